"""scopi_gpu_set_state: writing pos/q/v/omega back between steps (the reference's writable
container accessors, container.hpp:129,138,174,183, used between two ScopiSolver::run calls).

Bar: bit for bit.  Writing back the state just downloaded continues the run exactly as an
uninterrupted one; a changed velocity written through set_state continues exactly as the same
change written through set_particles (both keep the previous contacts).
"""
import numpy as np
import pytest

from gpu_helpers import gpu_solver
from scopi_b200 import configs
from scopi_b200.solver import ScopiGPUError

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "q", "v", "omega")


def _setup(side=8):
    pa = configs.spheres_1m(side=side)
    st = configs.SETTINGS["spheres_1m"]
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    return pa, kw, st["dt"]


def _state(s, pa):
    return s.download(pa.copy())


@pytest.mark.parametrize("precision", [0, 1])
def test_set_state_round_trip_continues_the_run(precision):
    pa, kw, dt = _setup()
    one = gpu_solver(pa, precision=precision, **kw)
    one.step(dt, 5)
    ref = _state(one, pa)
    two = gpu_solver(pa, precision=precision, **kw)
    two.step(dt, 3)
    mid = _state(two, pa)
    two.upload_state(mid)
    two.step(dt, 2)
    out = _state(two, pa)
    for k in FIELDS:
        assert np.array_equal(getattr(out, k), getattr(ref, k)), k
    assert np.array_equal(two.lagrange_multiplier(), one.lagrange_multiplier())


def test_set_state_matches_set_particles_after_a_change():
    pa, kw, dt = _setup()
    runs = []
    for use_state in (True, False):
        s = gpu_solver(pa, **kw)
        s.step(dt, 3)
        h = _state(s, pa)
        h.v[h.nb_inactive:] *= 0.5
        h.omega[h.nb_inactive:, 2] += 0.1
        (s.upload_state if use_state else s.upload)(h)
        s.step(dt, 2)
        runs.append((_state(s, pa), s.lagrange_multiplier()))
    (a, la), (b, lb) = runs
    for k in FIELDS:
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert np.array_equal(la, lb)


def test_set_state_writes_the_four_fields():
    pa, kw, dt = _setup(side=6)
    s = gpu_solver(pa, **kw)
    s.step(dt, 2)
    h = _state(s, pa)
    h.pos[h.nb_inactive:, 0] += 1e-4
    h.v[h.nb_inactive:, 1] += 1.0
    h.omega[h.nb_inactive:, 2] -= 2.0
    h.q[h.nb_inactive:] = [0.0, 0.0, 0.6, 0.8]
    s.upload_state(h)
    got = _state(s, pa)
    for k in FIELDS:
        assert np.array_equal(getattr(got, k), getattr(h, k)), k


def test_set_state_refuses_other_counts():
    pa, kw, dt = _setup(side=6)
    s = gpu_solver(pa, **kw)
    s.step(dt, 1)
    with pytest.raises(ScopiGPUError, match="must match"):
        s.upload_state(configs.spheres_1m(side=5))
    # the handle keeps working after the refusal
    s.step(dt, 1)
    assert np.isfinite(_state(s, pa).pos).all()
