"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the reference goldens.

Bar: contact lists identical and their geometry bit for bit on identical inputs;
trajectories within the reference's golden tolerances; FP64 positions within 1e-9
relative of the oracle step by step, multipliers within the solver tolerance (see
_trajectory for why the APGD iterate sequence can only be matched to rounding).
"""
import math

import numpy as np
import pytest

import scenes as S
from gpu_helpers import gpu_solver, oracle_solver, rel_err, same_contacts, segment_pile
from scopi_b200 import configs
from test_oracle_golden import APPROX, approx, compare_objects

pytestmark = pytest.mark.gpu


def detect_both(pa, **kw):
    g = gpu_solver(pa, **kw).detect()
    o = oracle_solver(pa, **kw).detect()
    return g, o


DETECT_SCENES = {
    "three_disks": lambda: (S.contacts_three_disks()[0], dict(kd_tree_radius=100.0)),
    "critical_2d": lambda: (S.critical_2d_spheres()[0], {}),
    "disks_2d_1024": lambda: (configs.disks_2d(), dict(dmax=0.01)),
    "box_3d_4000": lambda: (configs.box_3d(count=4000), dict(dmax=0.0045)),
    "spheres_16cube": lambda: (configs.spheres_1m(side=16), dict(dmax=0.0018)),
    "inclined_plane": lambda: (S.sphere_inclined_plane(math.pi / 6)[0], {}),
    "segment_pile": lambda: (segment_pile(), dict(dmax=0.009)),
    "kd_radius_filter": lambda: (configs.disks_2d(side=12), dict(dmax=0.05, kd_tree_radius=0.03 ** 2)),
    # rows of up to ~90 partners: past the search pass's per-row scratch (re-enumerated rows)
    "dense_rows": lambda: (configs.disks_2d(side=10), dict(dmax=0.2)),
}


@pytest.mark.parametrize("name", sorted(DETECT_SCENES))
@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
def test_contacts_bitexact(name, method):
    pa, kw = DETECT_SCENES[name]()
    g, o = detect_both(pa, contact_method=method, **kw)
    assert len(o["i"]) > 0
    same_contacts(g, o)


def test_contacts_three_disks_known_answer():
    """test/test_contacts_kdtree.cpp:14-73 on the GPU."""
    pa, kw, _, _ = S.contacts_three_disks()
    c = gpu_solver(pa, **kw).detect()
    assert list(c["i"]) == [0] and list(c["j"]) == [1]
    assert approx(c["dij"][0], math.sqrt(2.0) - 0.3)
    assert approx(c["nij"][0, 0], -1 / math.sqrt(2.0))


def test_matrix_known_values_and_adjoint():
    """test/test_matrices.cpp:17-77 on the GPU: A.u values and dot(Au, f) = dot(u, A^T f)."""
    pa, kw, _, _ = S.matrix_a_case2()
    s = gpu_solver(pa, **kw)
    s.detect()
    u = np.array([0.187562190766376, -1.184390935327111, 0., 0., 0., -0.00453709103433])
    sol = s.amat(u)
    assert approx(sol[0], -0.18595809) and approx(sol[1], 1.18278683)
    pa, kw, _, _ = S.matrix_a_3d()
    s = gpu_solver(pa, **kw)
    o = oracle_solver(pa, **kw)
    s.detect()
    o.detect()
    rng = np.random.default_rng(0)
    u = rng.random(12)
    f = rng.random(3)
    assert approx(float(np.dot(s.amat(u), f)), float(np.dot(u, s.atmat(f))))
    assert np.allclose(s.amat(u), o.amat(u), rtol=1e-14, atol=0)
    assert np.allclose(s.atmat(f), o.atmat(f), rtol=1e-14, atol=1e-300)


GOLDEN_CASES = [
    ("3spheres_nofriction", lambda: S.three_spheres(S.NOFRICTION), 1e-5),
    ("3spheres_viscous", lambda: S.three_spheres(S.VISCOUS), 1e-5),
    ("3spheres_friction_fp", lambda: S.three_spheres(S.FRICTION_FIXED_POINT), 1e-5),
    ("3spheres_viscous_friction", lambda: S.three_spheres(S.VISCOUS_FRICTION), 1e-5),
    ("sphere_plane_friction_mu01", S.sphere_plane_friction_mu01, 1e-5),
    ("two_spheres_asymmetrical", lambda: S.two_spheres(False), 1e-6),
    ("two_spheres_symmetrical", lambda: S.two_spheres(True), 1e-6),
    ("2d_case_spheres", S.critical_2d_spheres, 1e-6),
    ("obstacles_sphere_sphere_moving", lambda: S.obstacle_sphere_sphere("moving"), 1e-6),
]


@pytest.mark.parametrize("name,builder,tol", GOLDEN_CASES, ids=[c[0] for c in GOLDEN_CASES])
def test_reference_goldens_on_gpu(golden, name, builder, tol):
    pa, kw, dt, total = builder()
    s = gpu_solver(pa, **kw).run(dt, total)
    compare_objects(s.particles, golden[name]["objects"], 2, tol)


def test_critical_2d_contact_list_on_gpu(golden):
    """The 117-contact list of 2d_case_spheres.json, from the GPU state after 19 steps."""
    pa, kw, dt, total = S.critical_2d_spheres()
    s = gpu_solver(pa, **kw).run(dt, total - 1)
    c = s.detect()
    gold = golden["2d_case_spheres"]["contacts"]
    assert list(zip(c["i"].tolist(), c["j"].tolist())) == [(g["i"], g["j"]) for g in gold]
    for k, g in enumerate(gold):
        assert abs(c["dij"][k] - g["distance"]) < 1e-6


@pytest.mark.parametrize("alpha,e_pos,e_v", [(math.pi / 6, 0.000998789, 0.0010002),
                                             (math.pi / 4, 0.00100008, 0.00100119),
                                             (math.pi / 3, 0.00100105, 0.0010027)])
def test_inclined_plane_pinned_errors_on_gpu(alpha, e_pos, e_v):
    """test/test_obstacles.cpp:252-311 pinned errors, on the GPU."""
    pa, kw, dt, total = S.sphere_inclined_plane(alpha)
    s = gpu_solver(pa, **kw).run(dt, total)
    x, theta, v = S.analytic_inclined(alpha, 0.0, dt * (total + 1), 1.0, 1.0, 2.0)
    err_pos = np.linalg.norm(s.particles.pos[1, :2] - x) / np.linalg.norm(x)
    err_v = np.linalg.norm(s.particles.v[1, :2] - v) / np.linalg.norm(v)
    assert approx(err_pos, e_pos)
    assert abs(err_v - e_v) <= 1e-4 * (1 + e_v)


def test_viscous_analytic_on_gpu():
    """test/test_gradient.cpp:82-154 on the GPU (gamma carried across two run() calls)."""
    pa, kw, dt, total = S.sphere_plane_analytic(S.VISCOUS)
    s = gpu_solver(pa, **kw)
    s.run(dt, total)
    g, alpha = 1.0, math.pi / 4
    p2 = s.particles.copy()
    p2.f[1, :2] = (-g * math.sin(alpha), g * math.cos(alpha))
    s.set_particles(p2)
    s.run(dt, 500)
    x, v = S.analytic_viscous(alpha, dt * (total + 500), 1.0, g, 2.0, -2.0, dt * total)
    assert np.linalg.norm(s.particles.pos[1, :2] - x) / np.linalg.norm(x) <= 1e-3
    assert np.linalg.norm(s.particles.v[1, :2] - v) / np.linalg.norm(v) <= 1e-3


def _trajectory(pa, kw, dt, steps):
    """Step both engines from the same state and compare after every step.

    The backtracking test of apgd.hpp:174-175 compares two objective values that agree
    to rounding once the iterates have converged, so which branch it takes there is
    decided by rounding (the reference's own result depends on its BLAS), and a few
    hundred momentum iterations amplify rounding differences.  Bar: positions within
    1e-9 relative, velocities 1e-7; lambda within 1e-7 relative on steps whose branch
    trace (iterations, backtracks, restarts) is identical, and everywhere within the
    solver tolerance, |dlambda| <= 50 tol and 1e-6 relative.
    """
    g = gpu_solver(pa, **kw)
    o = oracle_solver(pa, **kw)
    tol = kw.get("tolerance", 1e-7)
    worst = {"lambda_same_trace": 0.0, "lambda_abs": 0.0, "lambda_rel": 0.0, "pos": 0.0, "v": 0.0, "same_trace": 0}
    for k in range(steps):
        g.run(dt, 1)
        o.run(dt, 1)
        gc, oc = g.current_contacts(), o.contacts()
        assert np.array_equal(gc["i"], oc["i"]) and np.array_equal(gc["j"], oc["j"]), f"contact pairs differ at step {k}"
        lg, lo = g.lagrange_multiplier(), o.lagrange_multiplier()
        assert len(lg) == len(lo)
        gs, os_ = g.stats(), o.stats()
        same = all(gs[x] == os_[x] for x in ("iterations", "backtracks", "restarts"))
        if len(lo):
            r = rel_err(lg, lo)
            if same:
                worst["same_trace"] += 1
                worst["lambda_same_trace"] = max(worst["lambda_same_trace"], r)
            worst["lambda_rel"] = max(worst["lambda_rel"], r)
            worst["lambda_abs"] = max(worst["lambda_abs"], float(np.linalg.norm(lg - lo)))
        worst["pos"] = max(worst["pos"], rel_err(g.particles.pos, o.pa.pos))
        worst["v"] = max(worst["v"], rel_err(g.particles.v, o.pa.v))
        assert abs(gs["iterations"] - os_["iterations"]) <= max(10, os_["iterations"] // 20)
    assert worst["lambda_same_trace"] <= 1e-7, worst
    assert worst["lambda_abs"] <= 50 * tol and worst["lambda_rel"] <= 1e-6, worst
    return worst


@pytest.mark.parametrize("name", ["disks_2d", "box_3d", "spheres", "spheres_viscous"])
def test_fp64_trajectory_matches_oracle(name):
    if name == "disks_2d":
        pa, st, steps = configs.disks_2d(), configs.SETTINGS["disks_2d"], 10
        kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    elif name == "box_3d":
        pa, st, steps = configs.box_3d(count=2000), configs.SETTINGS["box_3d"], 5
        kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    else:
        pa, st, steps = configs.spheres_1m(side=12), configs.SETTINGS["spheres_1m"], 5
        kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
        if name == "spheres_viscous":
            kw["problem"] = S.VISCOUS
    worst = _trajectory(pa, kw, st["dt"], steps)
    assert worst["pos"] <= 1e-9 and worst["v"] <= 1e-7, worst


def test_mixed_precision_reaches_violation_target():
    pa = configs.spheres_1m(side=16)
    st = configs.SETTINGS["spheres_1m"]
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    f64 = gpu_solver(pa, **kw).run(st["dt"], 3)
    mix = gpu_solver(pa, precision=1, mixed_violation_tol=1e-6, **kw).run(st["dt"], 3)
    sm = mix.stats()
    assert sm["violation"] <= 1e-6, sm
    assert sm["fp32_iterations"] > 0
    lam_err = rel_err(mix.lagrange_multiplier(), f64.lagrange_multiplier())
    assert lam_err <= 1e-2, lam_err
    assert rel_err(mix.particles.pos, f64.particles.pos) <= 1e-7


def test_mixed_fp64_correction_when_fp32_corrections_run_out():
    """No FP32 correction allowed and a target of 0 (never met): one correction runs in FP64
    (torque-free kernel with the offset) and ends at the FP64 solve's accuracy."""
    pa = configs.spheres_1m(side=16)
    st = configs.SETTINGS["spheres_1m"]
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    f64 = gpu_solver(pa, **kw).run(st["dt"], 3)
    mix = gpu_solver(pa, precision=1, mixed_violation_tol=0.0, mixed_max_corrections=0, **kw).run(st["dt"], 3)
    sm = mix.stats()
    assert sm["corrections"] == 1 and sm["violation"] <= max(1e-10, 10 * f64.stats()["violation"]), sm
    assert rel_err(mix.particles.pos, f64.particles.pos) <= 1e-7


def test_deterministic_bitwise():
    pa = configs.spheres_1m(side=12)
    st = configs.SETTINGS["spheres_1m"]
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    a = gpu_solver(pa, **kw).run(st["dt"], 3)
    b = gpu_solver(pa, **kw).run(st["dt"], 3)
    assert np.array_equal(a.particles.pos, b.particles.pos)
    assert np.array_equal(a.lagrange_multiplier(), b.lagrange_multiplier())


def test_kernel_launch_count_reported():
    pa = configs.disks_2d(side=8)
    s = gpu_solver(pa, dmax=0.01).run(0.005, 2)
    assert s.kernel_launches() > 0


def test_apgd_max_ite_reports_nonconvergence():
    pa = configs.disks_2d(side=8)
    s = gpu_solver(pa, dmax=0.01, max_ite=1, tolerance=1e-30)
    s.run(0.005, 1)
    st = s.stats()
    assert st["iterations"] == 1 and st["converged"] == 0 and st["status"] == 1


@pytest.mark.parametrize("precision,init", [(0, 1), (1, 0)])
def test_initial_step_choices(precision, init):
    """The first-step rule taken apart from the precision: FP64 with the curvature start and
    MIXED with the reference's alpha both reach the same state as the FP64 drop-in."""
    pa = configs.spheres_1m(side=16)
    st = configs.SETTINGS["spheres_1m"]
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    ref = gpu_solver(pa, **kw).run(st["dt"], 3)
    alt = gpu_solver(pa, precision=precision, initial_step=init, mixed_violation_tol=1e-6, **kw).run(st["dt"], 3)
    sa, sr = alt.stats(), ref.stats()
    assert sa["converged"] == 1 and sa["violation"] <= 1e-6, sa
    if init == 1:
        assert sa["iterations"] < sr["iterations"] / 4, (sa, sr)
    assert rel_err(alt.particles.pos, ref.particles.pos) <= 1e-7


@pytest.mark.parametrize("precision", [0, 1])
def test_friction_fixed_point_sphere_plane(precision):
    """FrictionFixedPoint on the reference's analytic case (test/test_gradient.cpp:215-283):
    the reference's error bounds against the rolling solution, and (FP64) the oracle's
    trajectory, which runs the same fixed-point loop."""
    import math

    from test_oracle_golden import fixed_point_errors
    pa, kw, dt, total = S.sphere_plane_fixed_point()
    g = gpu_solver(pa, precision=precision, **kw).run(dt, total)
    e_pos, e_q, e_v, e_om = fixed_point_errors(g.particles, dt, total)
    assert e_pos <= 1e-2 and e_q <= 1e-2, (e_pos, e_q)
    assert e_v <= 1.2e-5 and e_om <= 1.2e-5, (e_v, e_om)
    assert g.stats()["fixed_point_iterations"] >= 2
    if precision == 0:
        o = oracle_solver(pa, **kw).run(dt, total)
        assert rel_err(g.particles.pos, o.pa.pos) <= 1e-7
        assert rel_err(g.particles.v, o.pa.v) <= 1e-5
        assert math.isclose(g.particles.omega[1, 2], o.pa.omega[1, 2], rel_tol=1e-5)


@pytest.mark.parametrize("precision", [0, 1])
def test_viscous_friction_sphere_plane(precision):
    """ViscousFriction on the reference's analytic case (test/test_gradient.cpp:284-372): 500
    steps, the force flipped, 100 more; the reference's bounds (pos, q 1e-1; v, omega 1e-3) and
    (FP64) the oracle's trajectory, which runs the same fixed-point loop."""
    from test_oracle_golden import viscous_friction_errors
    pa, kw, dt, total = S.sphere_plane_viscous_friction()
    g = gpu_solver(pa, precision=precision, **kw)
    g.run(dt, total)
    p2 = g.particles.copy()
    p2.f[1, :2] = (-math.sin(math.pi / 4), math.cos(math.pi / 4))
    g.set_particles(p2)
    g.run(dt, 100)
    e_pos, e_q, e_v, e_om = viscous_friction_errors(g.particles, dt, total, 100)
    assert e_pos <= 1e-1 and e_q <= 1e-1, (e_pos, e_q)
    assert e_v <= 1e-3 and e_om <= 1e-3, (e_v, e_om)
    if precision == 0:
        o = oracle_solver(pa, **kw)
        o.run(dt, total)
        q2 = o.pa.copy()
        q2.f[1, :2] = (-math.sin(math.pi / 4), math.cos(math.pi / 4))
        o.set_particles(q2)
        o.run(dt, 100)
        assert rel_err(g.particles.pos, o.pa.pos) <= 1e-7
        assert rel_err(g.particles.v, o.pa.v) <= 1e-5
        assert math.isclose(g.particles.omega[1, 2], o.pa.omega[1, 2], rel_tol=1e-5, abs_tol=1e-9)


def viscous_friction_3d_deviations(steps=None):
    """Step the GPU (FP64) and the oracle together on the 3D ViscousFriction scene; the contact
    pairs and the modes (gamma at gamma_min, and the multipliers' row count in the reference's
    layout) must agree on every step; returns the worst deviations and the modes seen."""
    pa, kw, dt, total = S.viscous_friction_3d()
    g = gpu_solver(pa, **kw)
    o = oracle_solver(pa, **kw)
    seen = set()
    worst = {"gamma": 0.0, "lambda_rel": 0.0, "pos": 0.0, "v": 0.0}
    gmin = kw["gamma_min"]
    for k in range(total if steps is None else steps):
        g.run(dt, 1)
        o.run(dt, 1)
        gc, oc = g.current_contacts(), o.contacts()
        assert np.array_equal(gc["i"], oc["i"]) and np.array_equal(gc["j"], oc["j"]), k
        for gam in oc["gamma"]:
            seen.add(0 if gam >= -kw["gamma_tol"] else (2 if gam == gmin else 1))
        assert np.array_equal(gc["gamma"] == gmin, oc["gamma"] == gmin), k
        lg, lo = g.lagrange_multiplier(), o.lagrange_multiplier()
        assert len(lg) == len(lo), k
        assert g.stats()["fixed_point_iterations"] >= 1
        worst["gamma"] = max(worst["gamma"], float(np.max(np.abs(gc["gamma"] - oc["gamma"]))))
        worst["lambda_rel"] = max(worst["lambda_rel"], float(np.linalg.norm(lg - lo) / (1 + np.linalg.norm(lo))))
        worst["pos"] = max(worst["pos"], rel_err(g.particles.pos, o.pa.pos))
        worst["v"] = max(worst["v"], rel_err(g.particles.v, o.pa.v))
    return worst, seen


def test_viscous_friction_3d_matches_oracle():
    """ViscousFriction in 3D with all three multiplier layouts live (normal, viscous pair,
    gamma_min with the friction cone), FP64 against the oracle step by step.  The multipliers
    agree to the solver's accuracy (APGD tolerance 1e-7, a few solves per step), gamma
    accumulates dt n.lambda of each step (40 steps of dt 0.01), positions and velocities
    follow."""
    worst, seen = viscous_friction_3d_deviations()
    assert seen == {0, 1, 2}, seen
    assert worst["lambda_rel"] <= 1e-5 and worst["gamma"] <= 1e-7, worst
    assert worst["pos"] <= 1e-7 and worst["v"] <= 1e-5, worst


def test_viscous_friction_3d_mixed_precision():
    """The mixed path (FP32 iterations, FP64 corrections) on the same 3D scene: the
    trajectory of the FP64 solve within the FP32 solves' accuracy."""
    pa, kw, dt, total = S.viscous_friction_3d()
    f64 = gpu_solver(pa, **kw).run(dt, total)
    mix = gpu_solver(pa, precision=1, mixed_violation_tol=1e-6, **kw).run(dt, total)
    assert rel_err(mix.particles.pos, f64.particles.pos) <= 1e-6
    assert rel_err(mix.particles.v, f64.particles.v) <= 1e-3


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
def test_two_worms_on_gpu(golden, method):
    """test/test_worm.cpp:480-530 on the GPU: two_worms.json within its 1e-6, the final contact
    list (sorted pairs, then the glued links with normal and distance negated) equal to the
    reference's, and the trajectory of the oracle, which appends the same links."""
    from test_oracle_golden import compare_worms
    pa, kw, dt, total = S.two_worms(method)
    g = gpu_solver(pa, **kw).run(dt, total)
    compare_worms(g.particles, golden["two_worms"]["objects"], 2, 1e-6)
    c = g.current_contacts()
    gold = golden["two_worms"]["contacts"]
    assert list(zip(c["i"].tolist(), c["j"].tolist())) == [(x["i"], x["j"]) for x in gold]
    for k, x in enumerate(gold):
        assert abs(c["dij"][k] - x["distance"]) < 1e-6
        assert max(abs(c["nij"][k, d] - x["normal"][d]) for d in range(2)) < 1e-6
    o = oracle_solver(pa, **kw).run(dt, total)
    assert rel_err(g.particles.pos, o.pa.pos) <= 1e-9
    assert rel_err(g.particles.v, o.pa.v) <= 1e-6


def test_worms_need_nofriction_on_gpu():
    from scopi_b200 import ScopiGPUError
    pa, kw, dt, _ = S.two_worms()
    with pytest.raises(ScopiGPUError):
        gpu_solver(pa, **dict(kw, problem=S.FRICTION)).run(dt, 1)


def test_periodic_two_disks_on_gpu():
    """Periodic BoxDomain: the two disks meeting across the bound follow the oracle, and the
    same disks side by side without a box, modulo the period."""
    pa, kw, dt, total = S.periodic_two_disks()
    g = gpu_solver(pa, **kw)
    o = oracle_solver(pa, **kw)
    pu, kwu, _, _ = S.periodic_two_disks(unwrapped=True)
    u = gpu_solver(pu, **kwu)
    same_contacts(g.detect(), o.detect())
    for _ in range(total):
        g.run(dt, 1)
        o.run(dt, 1)
        u.run(dt, 1)
        gc, oc = g.current_contacts(), o.contacts()
        assert np.array_equal(gc["i"], oc["i"]) and np.array_equal(gc["j"], oc["j"])
        assert np.max(np.abs(g.particles.pos - o.pa.pos)) <= 1e-8
        dx = (g.particles.pos[:, 0] - u.particles.pos[:, 0]) % 4.0
        assert np.all(np.minimum(dx, 4.0 - dx) <= 1e-8)


@pytest.mark.parametrize("problem", [S.NOFRICTION, S.FRICTION, S.VISCOUS])
@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
def test_periodic_disks_match_oracle(problem, method):
    """Rows of disks crossing a periodic bound, GPU (FP64) against the oracle: on the same
    input the contact lists (copies mapped back to their bodies, closest points moved by the
    period, sorted by (i, j) with i > j across the bound) are equal bit for bit; stepped
    together, the pairs of every step and the trajectories agree."""
    pa, kw, dt, total = S.periodic_disks(problem, method)
    g = gpu_solver(pa, **kw)
    o = oracle_solver(pa, **kw)
    same_contacts(g.detect(), o.detect())
    across = 0
    for k in range(total):
        g.run(dt, 1)
        o.run(dt, 1)
        gc, oc = g.current_contacts(), o.contacts()
        assert np.array_equal(gc["i"], oc["i"]) and np.array_equal(gc["j"], oc["j"]), k
        # viscous gamma carried over by the mapped (i, j), pairs across the bound included
        assert np.max(np.abs(gc["gamma"] - oc["gamma"]), initial=0.0) <= 1e-7, k
        across += int(np.sum(gc["i"] > gc["j"]))
    assert across > 0
    assert rel_err(g.particles.pos, o.pa.pos) <= 1e-9
    assert rel_err(g.particles.v, o.pa.v) <= 1e-6


def test_periodic_mixed_precision():
    pa, kw, dt, total = S.periodic_disks()
    f64 = gpu_solver(pa, **kw).run(dt, total)
    mix = gpu_solver(pa, precision=1, mixed_violation_tol=1e-6, **dict(kw, tolerance=1e-7)).run(dt, total)
    assert mix.stats()["violation"] <= 1e-6
    assert rel_err(mix.particles.pos, f64.particles.pos) <= 1e-5


def test_periodic_obstacle_near_bound_rejected():
    from scopi_b200 import ScopiGPUError
    pa, kw, dt, _ = S.periodic_disks()
    pa.pos[0, 0] = 0.1
    with pytest.raises(ScopiGPUError):
        gpu_solver(pa, **kw).run(dt, 1)


@pytest.mark.parametrize("problem", [S.NOFRICTION, S.FRICTION])
def test_periodic_spheres_3d_match_oracle(problem):
    """The 3D periodic box (one periodic axis, floor plane): the same contact list bit for bit
    on the same input, the same pairs every step and the oracle's trajectory."""
    pa, kw, dt, total = S.periodic_spheres_3d(problem)
    g = gpu_solver(pa, **kw)
    o = oracle_solver(pa, **kw)
    same_contacts(g.detect(), o.detect())
    across = 0
    for k in range(total):
        g.run(dt, 1)
        o.run(dt, 1)
        gc, oc = g.current_contacts(), o.contacts()
        assert np.array_equal(gc["i"], oc["i"]) and np.array_equal(gc["j"], oc["j"]), k
        across += int(np.sum(gc["i"] > gc["j"]))
    assert across > 0
    assert rel_err(g.particles.pos, o.pa.pos) <= 1e-9
    assert np.all(g.particles.pos[1:, 0] >= 0.0) and np.all(g.particles.pos[1:, 0] <= 2.0)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["two_spheres_asymmetrical_friction", "2d_case_spheres_friction"])
def test_friction_goldens_on_gpu(golden, name, precision):
    """test/test_friction.cpp:17-112 on the GPU (the Friction rows of the 6-dof kernel), FP64
    and mixed, against the reference's snapshots (tol 1e-6)."""
    from test_oracle_golden import compare_positions
    pa, kw, dt, total = S.two_spheres_friction() if name.startswith("two") else S.critical_2d_spheres_friction()
    g = gpu_solver(pa, precision=precision, **kw).run(dt, total)
    compare_positions(g.particles, golden[name]["objects"], 2, 1e-6)
