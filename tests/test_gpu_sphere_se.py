"""Scenes of spheres and superellipsoids together on the GPU against the oracle: the
sphere-superellipsoid pairs (the reference's damped Newton method, closest_points.hpp:944-1463,
utils.hpp:81-118; pairs whose Newton result the acceptance test refuses are solved as two
superellipsoids) and the 2D superellipsoid-plane pairs (closed form, :1783-1958).

Contact lists: the same (i, j) pairs.  Geometry: sphere-sphere and sphere-plane rows bit for
bit (the same formulas, no contraction); the rows of superellipsoids within bounds stated by
how the oracle's solve of the row ended (BOUNDS): the GPU's and the host's pow / sin / cos
differ in the last bits, and the solves' stopping tests can turn on those bits.
"""
import numpy as np
import pytest

import py_oracle as orc
from gpu_helpers import gpu_solver, oracle_solver, rel_err
from mixed_scenes import mixed_box_2d, mixed_pile_3d

pytestmark = pytest.mark.gpu

SPHERE, PLANE, SEGMENT, SE = 0, 1, 2, 3

# Bounds of |GPU - oracle| on the rows of superellipsoids, relative to the bodies' size, by
# how the oracle's solve of the row ended (distance, points, normal).  Every solve stops near
# a double root of F3, where the distance is stationary and the points and normal are not,
# so the distance agrees far better than the points.  "newton": the Newton result kept (both
# engines stop on |d| < 1e-7 or |F| < 1e-10; at unit size |F| ~ 5e-4 x the squared angle
# error near the double root, so the stop leaves the angles ~5e-4 apart).  "converged": the hybrid method's info 1 (its
# step below xtol relative to the angles), or a closed form.  "stopped": the hybrid method's
# other stops (2: maxfev, 4 and 5: slow progress), whose result moves with the last bit of
# the inputs (the one-ulp sensitivity of tests/test_gpu_superellipsoid.py).
BOUNDS = {"newton": (1e-8, 1e-3, 5e-3), "converged": (1e-5, 1e-3, 2e-2), "stopped": (1e-2, 5e-2, 0.2)}


def _kinds(pa, c):
    sh = np.asarray(pa.shape)
    a, b = sh[c["i"]], sh[c["j"]]
    return np.minimum(a, b), np.maximum(a, b)


def _dim(pa):
    return 3 if np.any(np.asarray(pa.axes)[:, 2] > 0) else 2


def _record(pa, b):
    if int(pa.shape[b]) == SE:
        return orc.se_record(pa.pos[b], pa.q[b], pa.axes[b], pa.squareness[b])
    return orc.sphere_record(pa.pos[b], pa.q[b], pa.radius[b])


def _status(pa, i, j):
    """How the oracle's solve of row (i, j) ends: ('newton', iterations) when the Newton result
    is kept, ('hybrid', info) for the hybrid method of the superellipsoid pairs, None for the
    closed forms (superellipsoid-plane)."""
    si, sj = int(pa.shape[i]), int(pa.shape[j])
    if si == PLANE or sj == PLANE:
        return None
    dim = _dim(pa)
    if si == SE and sj == SE:
        f = orc.se_se if dim == 3 else orc.se2_se2
        return "hybrid", f(_record(pa, i), _record(pa, j))["info"]
    e, s = (i, j) if si == SE else (j, i)
    st = orc.sphere_se(dim, _record(pa, e), _record(pa, s), reference_labels=False, se_is_i=si == SE)["newton"]
    return ("newton", st) if st < 100 else ("hybrid", st - 100)


def _compare(pa, gc, oc, size):
    assert np.array_equal(gc["i"], oc["i"]) and np.array_equal(gc["j"], oc["j"]), "contact pairs differ"
    lo, hi = _kinds(pa, oc)
    exact = hi != SE  # sphere-sphere, sphere-plane
    for k in ("dij", "nij", "pi", "pj"):
        assert np.array_equal(gc[k][exact], oc[k][exact]), k
    count = {"newton": 0, "hybrid": 0, "closed form": 0}
    worst = {c: [0.0, 0.0, 0.0] for c in BOUNDS}
    for k in np.flatnonzero(~exact):
        st = _status(pa, int(oc["i"][k]), int(oc["j"][k]))
        if st is None:
            cls = "converged"
            count["closed form"] += 1
        else:
            count[st[0]] += 1
            cls = "newton" if st[0] == "newton" else ("converged" if st[1] == 1 else "stopped")
        e = [abs(gc["dij"][k] - oc["dij"][k]), float(np.max(np.abs(gc["pi"][k] - oc["pi"][k]))),
             float(np.max(np.abs(gc["nij"][k] - oc["nij"][k])))]
        worst[cls] = [max(a, b) for a, b in zip(worst[cls], e)]
        bd, bp, bn = BOUNDS[cls]
        assert e[0] <= bd * size and e[1] <= bp * size and e[2] <= bn, (k, st, e)
    print(f"rows {len(oc['i'])}: exact {int(exact.sum())}, {count}; worst |d dij|, |d p|, |d n| "
          f"(size {size}): {worst}")
    return count


@pytest.mark.parametrize("side,seed", [(5, 3), (7, 4)])
def test_mixed_pile_3d_contacts_match_the_oracle(side, seed):
    """Bodies of 4-8 mm: the reference's stopping test |F| < 1e-10 is absolute and F scales as
    a length to the fifth, so its Newton method stops at its start sample and the acceptance
    test refuses that result on every row: the rows all go to the hybrid method."""
    pa = mixed_pile_3d(side, seed)
    gc = gpu_solver(pa, dmax=0.004).detect()
    oc = oracle_solver(pa, dmax=0.004).detect()
    count = _compare(pa, gc, oc, 0.01)
    assert count["hybrid"] > 10


def test_mixed_pile_3d_unit_scale_contacts_match_the_oracle():
    """The same kind of pile at 25 times the size (bodies of 0.1-0.2, as in the reference's
    own closest-point tests): there the Newton result is kept on part of the rows."""
    pa = mixed_pile_3d(6, 11, scale=25.0)
    gc = gpu_solver(pa, dmax=0.1).detect()
    oc = oracle_solver(pa, dmax=0.1).detect()
    count = _compare(pa, gc, oc, 0.25)
    assert count["newton"] > 5


def test_mixed_box_2d_contacts_match_the_oracle():
    pa = mixed_box_2d(10, 5)
    gc = gpu_solver(pa, dmax=0.004).detect()
    oc = oracle_solver(pa, dmax=0.004).detect()
    lo, hi = _kinds(pa, oc)
    assert np.any((lo == PLANE) & (hi == SE)), "no superellipsoid-plane row"
    count = _compare(pa, gc, oc, 0.01)
    assert count["newton"] + count["hybrid"] > 3


def test_mixed_pile_3d_steps_match_the_oracle():
    """27 bodies falling on the floor, NoFriction, 60 steps on both engines from the same
    state: contact lists equal at every step; positions and velocities at the end within the
    stated bounds."""
    pa = mixed_pile_3d(3, 8)
    kw = dict(dmax=0.004, tolerance=1e-9, max_ite=20000)
    g = gpu_solver(pa, **kw)
    o = oracle_solver(pa, **kw)
    dt = 2e-3
    for k in range(60):
        g.run(dt, 1)
        o.run(dt, 1)
        gc, oc = g.current_contacts(), o.contacts()
        assert np.array_equal(gc["i"], oc["i"]) and np.array_equal(gc["j"], oc["j"]), k
    ep, ev = rel_err(g.particles.pos, o.pa.pos), rel_err(g.particles.v, o.pa.v)
    print("contacts", len(gc["i"]), "positions", ep, "velocities", ev)
    assert len(gc["i"]) >= 5
    assert ep <= 1e-7 and ev <= 1e-4
    g.close()


def test_superellipsoid_scenes_refuse_other_obstacles_and_worms():
    from scopi_b200 import _abi
    from scopi_b200.container import Particles, Property
    from scopi_b200.solver import ScopiGPUError
    cases = []
    p = Particles(2)  # superellipsoid-segment: unimplemented in the reference (closest_points.hpp:919-931)
    p.add_segment((0.0, 0.0), (0.2, 0.0))
    p.add_superellipsoid((0.0, 0.02), (0.01, 0.005), [1.0], Property())
    cases.append(p.finalize())
    p = Particles(3)  # a sphere obstacle
    p.add_sphere((0.0, 0.0, 0.0), 0.01, Property().deactivate())
    p.add_superellipsoid((0.0, 0.0, 0.03), (0.01, 0.005, 0.005), (1.0, 1.0), Property())
    cases.append(p.finalize())
    p = Particles(3)  # a worm beside a superellipsoid
    p.add_worm([(0.0, 0.0, 0.0), (0.02, 0.0, 0.0)], 0.01, Property())
    p.add_superellipsoid((0.0, 0.0, 0.05), (0.01, 0.005, 0.005), (1.0, 1.0), Property())
    cases.append(p.finalize())
    for pa in cases:
        with pytest.raises(ScopiGPUError) as exc:
            gpu_solver(pa, dmax=0.004).detect()
        assert f"({_abi.EUNSUPPORTED})" in str(exc.value), str(exc.value)
