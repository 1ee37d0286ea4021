"""Pin the CPU oracle against the reference's own golden files and known answers.

Every case is a reference test (cited per test); tolerances are the reference's
(test/utils.hpp:16 tolerance=1e-6, test/test_gradient.cpp:19 tol=1e-5,
doctest::Approx relative 1.2e-5).  These run without a GPU.
"""
import math

import numpy as np
import pytest

import py_oracle as orc
import scenes as S

APPROX = 1.1920929e-07 * 100  # doctest::Approx default epsilon (FLT_EPSILON * 100)


def approx(a, b, eps=APPROX):
    return abs(a - b) <= eps * (1 + max(abs(a), abs(b)))


def run_oracle(scene, steps=None):
    pa, kw, dt, total = scene
    s = orc.OracleSolver(pa, **kw)
    s.run(dt, total if steps is None else steps)
    return s


def compare_objects(state, gold_objs, dim, tol):
    worst = 0.0
    for k, o in enumerate(gold_objs):
        for d in range(dim):
            worst = max(worst, abs(state.pos[k, d] - o["position"][d]))
            worst = max(worst, abs(state.v[k, d] - o["velocity"][d]))
        om = o["omega"]
        if dim == 2:
            worst = max(worst, abs(state.omega[k, 2] - om[0]))
        else:
            for d in range(3):
                worst = max(worst, abs(state.omega[k, d] - om[d]))
        for d in range(4):
            worst = max(worst, abs(state.q[k, d] - o["quaternion"][d]))
    assert worst <= tol, f"max abs deviation {worst:.3e} > {tol}"
    return worst


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
def test_contacts_three_disks(method):
    """test/test_contacts_kdtree.cpp:14-73, test/test_contacts_brute_force.cpp:12-71."""
    pa, kw, _, _ = S.contacts_three_disks()
    kw = dict(kw, contact_method=method)
    c = orc.OracleSolver(pa, **kw).detect()
    assert len(c["i"]) == 1 and c["i"][0] == 0 and c["j"][0] == 1
    assert approx(c["dij"][0], math.sqrt(2.0) - 0.1 - 0.2)
    assert approx(c["nij"][0, 0], -1 / math.sqrt(2.0)) and approx(c["nij"][0, 1], -1 / math.sqrt(2.0))
    assert approx(c["pi"][0, 0], 0.1 * math.sqrt(2.0) / 2.0) and approx(c["pi"][0, 1], 0.1 * math.sqrt(2.0) / 2.0)
    assert approx(c["pj"][0, 0], 1 - 0.2 * math.sqrt(2.0) / 2.0) and approx(c["pj"][0, 1], 1 - 0.2 * math.sqrt(2.0) / 2.0)


def test_matrix_a_adjoint():
    """test/test_matrices.cpp:17-45: dot(A u, f) == dot(u, A^T f)."""
    pa, kw, _, _ = S.matrix_a_3d()
    s = orc.OracleSolver(pa, **kw)
    s.detect()
    rng = np.random.default_rng(0)
    u = rng.random(6 * 2)
    f = rng.random(3 * 1)
    assert approx(float(np.dot(s.amat(u), f)), float(np.dot(u, s.atmat(f))))


def test_matrix_a_case2():
    """test/test_matrices.cpp:47-77: sphere on a 45-degree plane, known A.u values."""
    pa, kw, _, _ = S.matrix_a_case2()
    s = orc.OracleSolver(pa, **kw)
    c = s.detect()
    assert len(c["i"]) == 1
    u = np.array([0.187562190766376, -1.184390935327111, 0., 0., 0., -0.00453709103433])
    sol = s.amat(u)
    assert approx(sol[0], -0.18595809) and approx(sol[1], 1.18278683)


@pytest.mark.parametrize("name,problem", [("3spheres_nofriction", S.NOFRICTION), ("3spheres_viscous", S.VISCOUS),
                                          ("3spheres_friction_fp", S.FRICTION_FIXED_POINT),
                                          ("3spheres_viscous_friction", S.VISCOUS_FRICTION)])
def test_three_spheres_golden(golden, name, problem):
    """test/test_gradient.cpp:377-642 against test/references/3spheres_*.json (tol 1e-5)."""
    s = run_oracle(S.three_spheres(problem))
    compare_objects(s.pa, golden[name]["objects"], 2, 1e-5)


def test_sphere_plane_friction_golden(golden):
    """test/test_gradient.cpp:156-213 against sphere_plane_friction_mu01.json (tol 1e-5)."""
    s = run_oracle(S.sphere_plane_friction_mu01())
    compare_objects(s.pa, golden["sphere_plane_friction_mu01"]["objects"], 2, 1e-5)


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
@pytest.mark.parametrize("sym", [False, True])
def test_two_spheres_golden(golden, sym, method):
    """test/test_sphere.cpp:341-421 against two_spheres_*.json (tol 1e-6)."""
    s = run_oracle(S.two_spheres(sym, method))
    name = "two_spheres_symmetrical" if sym else "two_spheres_asymmetrical"
    compare_objects(s.pa, golden[name]["objects"], 2, 1e-6)


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
def test_critical_2d_golden(golden, method):
    """test/test_sphere.cpp:423-484 against 2d_case_spheres.json (tol 1e-6), with its contact list."""
    scene = S.critical_2d_spheres(method)
    s = run_oracle(scene, steps=scene[3] - 1)
    c = s.detect()  # the snapshot's contacts are those of the last step
    gold = golden["2d_case_spheres"]
    gi = [(g["i"], g["j"]) for g in gold["contacts"]]
    assert list(zip(c["i"].tolist(), c["j"].tolist())) == gi
    for k, g in enumerate(gold["contacts"]):
        assert abs(c["dij"][k] - g["distance"]) < 1e-6
        for d in range(2):
            assert abs(c["nij"][k, d] - g["normal"][d]) < 1e-6
            assert abs(c["pi"][k, d] - g["pi"][d]) < 1e-6
            assert abs(c["pj"][k, d] - g["pj"][d]) < 1e-6
    s = run_oracle(scene)
    compare_objects(s.pa, gold["objects"], 2, 1e-6)


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
@pytest.mark.parametrize("variant", ["fixed", "velocity", "force"])
def test_obstacle_sphere_plane(variant, method):
    """test/test_obstacles.cpp:14-98: the sphere stays at (0, 1) on plane(pi/2)."""
    s = run_oracle(S.obstacle_sphere_plane(variant, method))
    pos, q = s.pa.pos, s.pa.q
    assert approx(pos[0, 0], 0) and approx(pos[0, 1], 0) and approx(pos[1, 0], 0) and approx(pos[1, 1], 1)
    assert approx(q[0, 0], math.sqrt(2) / 2) and approx(q[0, 3], math.sqrt(2) / 2)
    assert approx(q[1, 0], 1) and approx(q[1, 3], 0)


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
@pytest.mark.parametrize("variant", ["fixed", "velocity", "force"])
def test_obstacle_sphere_sphere(variant, method):
    """test/test_obstacles.cpp:100-212: the sphere stays at (0, 2) on the fixed sphere."""
    s = run_oracle(S.obstacle_sphere_sphere(variant, method))
    pos, q = s.pa.pos, s.pa.q
    assert approx(pos[0, 0], 0) and approx(pos[0, 1], 0) and approx(pos[1, 0], 0) and approx(pos[1, 1], 2)
    assert approx(q[1, 0], 1) and approx(q[1, 3], 0)


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
def test_obstacle_sphere_sphere_moving(golden, method):
    """test/test_obstacles.cpp:214-250 against obstacles_sphere_sphere_moving.json (tol 1e-6)."""
    s = run_oracle(S.obstacle_sphere_sphere("moving", method))
    compare_objects(s.pa, golden["obstacles_sphere_sphere_moving"]["objects"], 2, 1e-6)


@pytest.mark.parametrize("alpha,e_pos,e_q,e_v", [(math.pi / 6, 0.000998789, 0.0, 0.0010002),
                                                  (math.pi / 4, 0.00100008, 0.0, 0.00100119),
                                                  (math.pi / 3, 0.00100105, 0.0, 0.0010027)])
def test_sphere_inclined_plane(alpha, e_pos, e_q, e_v):
    """test/test_obstacles.cpp:252-311: pinned relative errors against the analytic solution."""
    scene = S.sphere_inclined_plane(alpha)
    s = run_oracle(scene)
    dt, total = scene[2], scene[3]
    x, theta, v = S.analytic_inclined(alpha, 0.0, dt * (total + 1), 1.0, 1.0, 2.0)
    qa = S.quaternion(theta)
    pos = s.pa.pos[1, :2]
    err_pos = np.linalg.norm(pos - x) / np.linalg.norm(x)
    err_q = np.linalg.norm(s.pa.q[1] - qa) / np.linalg.norm(qa)
    err_v = np.linalg.norm(s.pa.v[1, :2] - v) / np.linalg.norm(v)
    assert approx(err_pos, e_pos)
    assert approx(err_q, e_q)
    assert abs(err_v - e_v) <= 1e-4 * (1 + max(abs(err_v), abs(e_v)))
    assert approx(s.pa.omega[1, 2], 0.0)


def test_sphere_plane_no_friction_analytic():
    """test/test_gradient.cpp:23-80: errors vs the analytic solution (pos/q 1e-3, v 1e-12)."""
    scene = S.sphere_plane_analytic(S.NOFRICTION)
    s = run_oracle(scene)
    t = scene[2] * scene[3]
    x, v = S.analytic_no_friction(math.pi / 4, t, 1.0, 1.0, 2.0)
    assert np.linalg.norm(s.pa.pos[1, :2] - x) / np.linalg.norm(x) <= 1e-3
    assert np.linalg.norm(s.pa.q[1] - S.quaternion(0.0)) <= 1e-3
    assert np.linalg.norm(s.pa.v[1, :2] - v) / np.linalg.norm(v) <= 1e-12 * (1 + APPROX)
    assert approx(s.pa.omega[1, 2], 0.0)


def test_sphere_plane_viscous_analytic():
    """test/test_gradient.cpp:82-154: two runs (force flipped), errors vs analytic (1e-3)."""
    pa, kw, dt, total = S.sphere_plane_analytic(S.VISCOUS)
    s = orc.OracleSolver(pa, **kw)
    s.run(dt, total)
    g, alpha = 1.0, math.pi / 4
    p2 = s.pa.copy()
    p2.f[1, :2] = (-g * math.sin(alpha), g * math.cos(alpha))
    s.set_particles(p2)
    s.run(dt, 500)
    x, v = S.analytic_viscous(alpha, dt * (total + 500), 1.0, g, 2.0, -2.0, dt * total)
    assert np.linalg.norm(s.pa.pos[1, :2] - x) / np.linalg.norm(x) <= 1e-3
    assert np.linalg.norm(s.pa.v[1, :2] - v) / np.linalg.norm(v) <= 1e-3
    assert approx(s.pa.omega[1, 2], 0.0)


def fixed_point_errors(pa, dt, total):
    """Errors of test/test_gradient.cpp:264-283 (relative norms; omega with std::norm, i.e. squared)."""
    x, theta, v, om = S.analytic_friction(math.pi / 4, 0.5, dt * total, 1.0, 1.0, 2.0)
    qa = S.quaternion(theta)
    e_pos = math.hypot(pa.pos[1, 0] - x[0], pa.pos[1, 1] - x[1]) / math.hypot(*x)
    e_q = float(np.linalg.norm(pa.q[1] - qa) / np.linalg.norm(qa))
    e_v = math.hypot(pa.v[1, 0] - v[0], pa.v[1, 1] - v[1]) / math.hypot(*v)
    e_om = (pa.omega[1, 2] - om) ** 2 / om ** 2
    return e_pos, e_q, e_v, e_om


def test_sphere_plane_friction_fixed_point_analytic():
    """test/test_gradient.cpp:215-283 (FrictionFixedPoint): pos and q within 1e-2 of the
    analytic rolling solution, v and omega within doctest::Approx of 1e-12."""
    pa, kw, dt, total = S.sphere_plane_fixed_point()
    s = orc.OracleSolver(pa, **kw)
    s.run(dt, total)
    e_pos, e_q, e_v, e_om = fixed_point_errors(s.pa, dt, total)
    assert e_pos <= 1e-2 and e_q <= 1e-2, (e_pos, e_q)
    assert approx(e_v, 1e-12) or e_v <= 1e-12, e_v
    assert approx(e_om, 1e-12) or e_om <= 1e-12, e_om
    assert s.stats()["fixed_point_iterations"] >= 2


def viscous_friction_errors(pa, dt, total, total2):
    """Errors of test/test_gradient.cpp:341-366 (relative norms; omega with std::norm)."""
    x, theta, v, om = S.analytic_viscous_friction(math.pi / 4, 0.5, dt * (total + total2), 1.0, 1.0, 2.0, -1.4,
                                                  dt * total)
    qa = S.quaternion(theta)
    e_pos = math.hypot(pa.pos[1, 0] - x[0], pa.pos[1, 1] - x[1]) / math.hypot(*x)
    e_q = float(np.linalg.norm(pa.q[1] - qa) / np.linalg.norm(qa))
    e_v = math.hypot(pa.v[1, 0] - v[0], pa.v[1, 1] - v[1]) / math.hypot(*v)
    e_om = (pa.omega[1, 2] - om) ** 2 / om ** 2
    return e_pos, e_q, e_v, e_om


def test_sphere_plane_viscous_friction_analytic():
    """test/test_gradient.cpp:284-372 (ViscousFriction): 500 steps, the force flipped, 100 more;
    pos and q within 1e-1 of the analytic solution, v and omega within 1e-3."""
    pa, kw, dt, total = S.sphere_plane_viscous_friction()
    s = orc.OracleSolver(pa, **kw)
    s.run(dt, total)
    p2 = s.pa.copy()
    p2.f[1, :2] = (-math.sin(math.pi / 4), math.cos(math.pi / 4))
    s.set_particles(p2)
    s.run(dt, 100)
    e_pos, e_q, e_v, e_om = viscous_friction_errors(s.pa, dt, total, 100)
    assert e_pos <= 1e-1 and e_q <= 1e-1, (e_pos, e_q)
    assert e_v <= 1e-3 * (1 + APPROX) and e_om <= 1e-3 * (1 + APPROX), (e_v, e_om)


def compare_worms(state, gold_objs, dim, tol):
    """The fields of a worm that test/utils.cpp:14-75 diffs: each sphere's position and
    quaternion, and the velocity and omega of the worm's first sphere."""
    worst, b = 0.0, 0
    for o in gold_objs:
        assert o["type"] == "worm"
        first = b
        for sph in o["spheres"]:
            assert sph["id"] == b
            for d in range(dim):
                worst = max(worst, abs(state.pos[b, d] - sph["position"][d]))
            for d in range(4):
                worst = max(worst, abs(state.q[b, d] - sph["quaternion"][d]))
            b += 1
        for d in range(dim):
            worst = max(worst, abs(state.v[first, d] - o["velocity"][d]))
        worst = max(worst, abs(state.omega[first, 2] - o["omega"][0]))
    assert b == state.n, (b, state.n)
    assert worst <= tol, f"max abs deviation {worst:.3e} > {tol}"
    return worst


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
def test_two_worms_golden(golden, method):
    """test/test_worm.cpp:480-530 against test/references/two_worms.json (tol 1e-6), and its
    final contact list: the contact method's sorted pairs, then one glued link per pair of
    consecutive spheres with normal and distance negated."""
    s = run_oracle(S.two_worms(method))
    compare_worms(s.pa, golden["two_worms"]["objects"], 2, 1e-6)
    c = s.contacts()
    gold = golden["two_worms"]["contacts"]
    assert list(zip(c["i"].tolist(), c["j"].tolist())) == [(g["i"], g["j"]) for g in gold]
    for k, g in enumerate(gold):
        assert abs(c["dij"][k] - g["distance"]) < 1e-6
        for d in range(2):
            assert abs(c["nij"][k, d] - g["normal"][d]) < 1e-6


def test_worms_need_nofriction():
    """Worm links carry the reference's default-constructed contact property; only the
    NoFriction problem, where the property is empty, is accepted."""
    pa, kw, _, _ = S.two_worms()
    with pytest.raises(RuntimeError):
        orc.OracleSolver(pa, **dict(kw, problem=S.FRICTION))


def test_periodic_two_disks_match_unwrapped():
    """BoxDomain periodic along x (box.hpp, utils.hpp:229-257, base.hpp:118-137,
    solver.hpp:482-522): two disks meeting across the bound move as the same two disks
    side by side without a box, positions equal modulo the period (to the solver's
    accuracy: the contact across the bound is listed as (B, A), the other as (A, B))."""
    pa, kw, dt, total = S.periodic_two_disks()
    s = orc.OracleSolver(pa, **kw)
    pu, kwu, _, _ = S.periodic_two_disks(unwrapped=True)
    u = orc.OracleSolver(pu, **kwu)
    met = False
    for _ in range(total):
        s.run(dt, 1)
        u.run(dt, 1)
        c = s.contacts()
        met = met or len(c["i"]) > 0
        for k in range(2):
            dx = (s.pa.pos[k, 0] - u.pa.pos[k, 0]) % 4.0
            assert min(dx, 4.0 - dx) <= 1e-8 and abs(s.pa.pos[k, 1] - u.pa.pos[k, 1]) <= 1e-8
            assert 0.0 <= s.pa.pos[k, 0] <= 4.0
    assert met
    # the disks stopped against each other across the bound: gap closed, not crossed
    gap = (s.pa.pos[0, 0] + 4.0 - s.pa.pos[1, 0]) - 0.5
    assert abs(gap) <= 1e-9, gap


def test_periodic_disks_invariants():
    """Rows of disks crossing the periodic bound: every body stays in the box, a contact
    across the bound has each closest point on its own body, and the x momentum (no
    external x force, frictionless floor) is kept."""
    pa, kw, dt, total = S.periodic_disks()
    s = orc.OracleSolver(pa, **kw)
    px0 = float(np.sum(s.pa.v[1:, 0] * s.pa.m[1:]))
    across = 0
    for _ in range(total):
        before = s.pa.pos.copy()  # the step's contacts are those of the positions it starts from
        s.run(dt, 1)
        assert np.all(s.pa.pos[1:, 0] >= 0.0) and np.all(s.pa.pos[1:, 0] <= 4.0)
        c = s.contacts()
        for k in range(len(c["i"])):
            i, j = int(c["i"][k]), int(c["j"][k])
            if i == 0:
                continue
            if abs(before[i, 0] - before[j, 0]) > 2.0:
                across += 1
                # pi on body i; pj found on the copy of body j and moved back by the period,
                # so on body j itself (the lever arm pj - x_j of the A matrix)
                assert abs(np.linalg.norm(c["pi"][k, :2] - before[i, :2]) - 0.2) <= 1e-12
                assert abs(np.linalg.norm(c["pj"][k, :2] - before[j, :2]) - 0.2) <= 1e-12
        px = float(np.sum(s.pa.v[1:, 0] * s.pa.m[1:]))
        assert abs(px - px0) <= 1e-7 * (1 + abs(px0)), (px, px0)
    assert across > 0


def test_periodic_obstacle_near_bound_fails():
    """An obstacle within dmax of a periodic lower bound: the reference copies it and pairs it
    with itself through the unimplemented plane-plane case; the oracle refuses the step."""
    pa, kw, dt, _ = S.periodic_disks()
    pa.pos[0, 0] = 0.1
    s = orc.OracleSolver(pa, **kw)
    with pytest.raises(RuntimeError):
        s.run(dt, 1)


def compare_positions(state, gold_objs, dim, tol):
    """Older snapshots hold no properties: positions and quaternions (test/utils.cpp:14-75)."""
    worst = 0.0
    for k, o in enumerate(gold_objs):
        worst = max(worst, max(abs(state.pos[k, d] - o["position"][d]) for d in range(dim)))
        worst = max(worst, max(abs(state.q[k, d] - o["quaternion"][d]) for d in range(4)))
    assert worst <= tol, f"max abs deviation {worst:.3e} > {tol}"
    return worst


@pytest.mark.parametrize("method", [S.KDTREE, S.BRUTE_FORCE])
@pytest.mark.parametrize("name", ["two_spheres_asymmetrical_friction", "2d_case_spheres_friction"])
def test_friction_goldens(golden, name, method):
    """test/test_friction.cpp:17-112 against their snapshots (tol 1e-6)."""
    scene = S.two_spheres_friction(method) if name.startswith("two") else S.critical_2d_spheres_friction(method)
    s = run_oracle(scene)
    compare_positions(s.pa, golden[name]["objects"], 2, 1e-6)
