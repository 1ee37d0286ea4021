"""The bounded grid-barrier wait of the persistent APGD launches, run out on purpose.

Every wait inside a persistent APGD launch has a limit (scopi_gpu_params.barrier_timeout_us,
20 s by default).  scopi_gpu_test_barrier_stall arms one launch in which block 0 does not
count its first arrival, so that barrier never completes: every block waits until the
limit (set to a few milliseconds here), sets the error word and returns.  The step must
fail with SCOPI_GPU_ETIMEOUT, the CUDA context must stay usable, and the same handle's next
step must give exactly the result of a fresh handle's first step (the failed step moved
nothing: walls are static and vap_fixed only sets v = v_desired).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _settings():
    from scopi_b200 import configs
    st = configs.SETTINGS["spheres_1m"]
    return dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"]), st["dt"]


@pytest.mark.parametrize("case", ["fp64_torque_free", "mixed_curvature_start", "fp64_friction_rows"])
def test_barrier_limit_runs_out_and_handle_recovers(case):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from scopi_b200 import FP64, FRICTION, MIXED, ScopiSolver, _abi, configs
    from scopi_b200.solver import ScopiGPUError
    kw, dt = _settings()
    if case == "mixed_curvature_start":
        kw["precision"] = MIXED
    elif case == "fp64_friction_rows":
        kw["problem"] = FRICTION  # the 6-dof kernel and its barrier
        kw["precision"] = FP64
    pa = configs.spheres_1m(side=8)
    s = ScopiSolver(pa, barrier_timeout_us=5000, **kw)
    s.step(dt, 0)  # creates the handle and uploads the particles
    lib = _abi.load()
    assert lib.scopi_gpu_test_barrier_stall(s._h) == 0
    with pytest.raises(ScopiGPUError) as exc:
        s.step(dt, 1)
    assert f"({_abi.ETIMEOUT})" in str(exc.value) and "timed out" in str(exc.value)
    # the context still works: a plain torch kernel and the library's next step
    x = torch.arange(16, device="cuda", dtype=torch.float64)
    assert float((x * 2).sum().item()) == 240.0
    assert s.step(dt, 1) in (0, _abi.ENOCONV)
    s.sync()
    ref = ScopiSolver(pa, **kw).run(dt, 1)
    assert np.array_equal(s.particles.pos, ref.particles.pos)
    assert np.array_equal(s.particles.v, ref.particles.v)
    assert s.stats()["status"] == 0
    s.close()
    ref.close()


def test_barrier_stall_refused_for_batches():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from scopi_b200 import ScopiBatch, _abi, configs
    st = configs.SETTINGS["pile_scenes"]
    b = ScopiBatch(configs.pile_scenes(2), vap=st["vap"], dmax=st["dmax"], tolerance=st["tolerance"],
                   max_ite=st["max_ite"])
    lib = _abi.load()
    assert lib.scopi_gpu_test_barrier_stall(b._h) == _abi.EINVAL
    assert b"grid barrier" in lib.scopi_gpu_last_error(b._h)
    b.close()
