"""bench.cpu_sample's extrapolation (host logic, CPU): two capped oracle steps give the cost
of an APGD iteration and the fixed cost of a step, and steps/s is rebuilt from them.  A fake
oracle with known costs stands in for the real one."""
import sys
import types

import pytest

SETUP, T_ITER, T_CONTACTS, T_OTHER = 0.7, 0.25, 1.5, 0.05


class _FakeSolver:
    def __init__(self, pa, max_ite, **kw):
        self.n = max_ite

    def run(self, dt, steps):
        pass

    def stats(self):
        return {"iterations": self.n, "seconds_solve": SETUP + T_ITER * self.n, "seconds_contacts": T_CONTACTS,
                "seconds_other": T_OTHER, "contacts": 42}


@pytest.fixture
def fake_oracle(monkeypatch):
    mod = types.ModuleType("py_oracle")
    mod.OracleSolver = _FakeSolver
    monkeypatch.setitem(sys.modules, "py_oracle", mod)


@pytest.mark.parametrize("caps", [(1, 3), (1, 20), (2, 7)])
def test_cpu_sample_recovers_the_costs(fake_oracle, caps):
    import bench
    r = bench.cpu_sample(None, 500, 1, solver=({}, 1e-3), caps=caps)
    assert r["t_per_iteration_s"] == pytest.approx(T_ITER, rel=1e-12)
    assert r["t_outside_apgd_s"] == pytest.approx(SETUP + T_CONTACTS + T_OTHER, rel=1e-12)
    assert r["value"] == pytest.approx(1.0 / (SETUP + T_CONTACTS + T_OTHER + T_ITER * 500), rel=1e-12)
    assert r["iterations_timed"] == caps[0] + caps[1] and r["contacts"] == 42


def test_cpu_sample_single_cap_is_an_upper_bound(fake_oracle):
    import bench
    r = bench.cpu_sample(None, 500, 1, solver=({}, 1e-3), caps=(3,))
    # the one capped solve's set-up is spread over its iterations: a slower (lower) estimate
    assert r["t_per_iteration_s"] == pytest.approx(T_ITER + SETUP / 3, rel=1e-12)
    assert r["value"] < 1.0 / (SETUP + T_CONTACTS + T_OTHER + T_ITER * 500)
