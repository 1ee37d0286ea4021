"""Batched ensemble (many independent 2D pile scenes, one persistent solve launch per step,
one CUDA graph replay per step) against each scene stepped alone: by the oracle (CPU
restatement of ScopiSolver, include/scopi/solver.hpp:153-178) and by the single-scene GPU
solver."""
import numpy as np
import pytest

from gpu_helpers import oracle_solver, rel_err
from scopi_b200 import FP64, FRICTION, MIXED, ScopiBatch, ScopiGPUError, ScopiSolver, configs
from scopi_b200.container import Particles, Property

pytestmark = pytest.mark.gpu

ST = configs.SETTINGS["pile_scenes"]
KW = dict(dmax=ST["dmax"], tolerance=ST["tolerance"], max_ite=ST["max_ite"])


def small_piles(n, nmin=30, nmax=300, seed=7, vmax=0.6):
    """Pile scenes whose disks start with random velocities in [-vmax, vmax]^2, so the
    first steps already have active constraints."""
    return configs.pile_scenes(n, seed, nmin, nmax, vmax)


def lone_disk():
    """A scene without contacts: one disk far above its segment (free fall)."""
    p = Particles(2)
    p.add_segment((0.0, 0.0), (0.5, 0.0))
    m = 1.3
    p.add_sphere((0.25, 0.8), 0.01, Property(mass=m, moment_inertia=0.5 * m * 1e-4, force=(0.0, -9.81 * m)))
    return p.finalize()


def test_batch_fp64_matches_oracle_per_scene():
    scenes = small_piles(4)
    steps = 8
    b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, **KW)
    oracles = [oracle_solver(s, vap=ST["vap"], **KW) for s in scenes]
    for k in range(steps):
        b.run(ST["dt"], 1)
        for s, o in enumerate(oracles):
            o.run(ST["dt"], 1)
            assert b.scene_stats(s)["contacts"] == len(o.contacts()["i"]), f"scene {s} step {k}"
    iters = 0
    for s, o in enumerate(oracles):
        g = b.scene(s)
        assert rel_err(g.pos, o.pa.pos) <= 1e-9, s
        assert rel_err(g.v, o.pa.v) <= 1e-7, s
        assert b.scene_stats(s)["converged"] == 1
        iters = max(iters, b.scene_stats(s)["iterations"])
    assert iters > 10  # the solves did work


def test_batch_fp64_matches_single_scene_gpu():
    scenes = small_piles(6, 100, 1500, seed=8) + [lone_disk()]
    steps = 6
    b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, **KW).run(ST["dt"], steps)
    for s, pa in enumerate(scenes):
        one = ScopiSolver(pa, vap=ST["vap"], precision=FP64, **KW).run(ST["dt"], steps)
        g = b.scene(s)
        assert b.scene_stats(s)["contacts"] == one.stats()["contacts"], s
        assert rel_err(g.pos, one.particles.pos) <= 1e-9, s
        assert rel_err(g.v, one.particles.v) <= 1e-7, s


def test_batch_scene_without_contacts_falls_freely():
    scenes = small_piles(2) + [lone_disk()]
    b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, **KW).run(ST["dt"], 5)
    st = b.scene_stats(2)
    assert st["contacts"] == 0 and st["iterations"] == 0
    g = b.scene(2)
    # vap_fpd: v_{k+1} = v_k + dt f/m, then x += dt v (solver.hpp:138-148, vap_fpd.hpp:26-38)
    v, y = 0.0, 0.8
    for _ in range(5):
        v += ST["dt"] * -9.81
        y += ST["dt"] * v
    assert abs(g.v[1, 1] - v) <= 1e-12 and abs(g.pos[1, 1] - y) <= 1e-12


def test_batch_mixed_reaches_violation_target():
    scenes = small_piles(6, 100, 1500, seed=9)
    f64 = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, **KW).run(ST["dt"], 3)
    mix = ScopiBatch(scenes, vap=ST["vap"], precision=MIXED, mixed_violation_tol=1e-6, **KW).run(ST["dt"], 3)
    for s in range(len(scenes)):
        st = mix.scene_stats(s)
        assert st["violation"] <= 1e-6, (s, st)
        if st["contacts"]:
            assert st["fp32_iterations"] > 0
        assert rel_err(mix.scene(s).pos, f64.scene(s).pos) <= 1e-7, s


def test_batch_block_sizes_agree_and_are_deterministic():
    scenes = small_piles(5, 100, 1500, seed=10)
    runs = {}
    for bt in (256, 1024, 256):
        b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, block_threads=bt, **KW).run(ST["dt"], 4)
        assert b.block_threads() == bt
        pos = [b.scene(s).pos.copy() for s in range(len(scenes))]
        if bt in runs:
            for a, c in zip(runs[bt], pos):
                assert np.array_equal(a, c), "same block size, different result"
        runs[bt] = pos
    for a, c in zip(runs[256], runs[1024]):
        assert rel_err(a, c) <= 1e-9


@pytest.mark.parametrize("threads,tile", [(256, 2), (512, 2), (1024, 2), (512, 1), (2048, 1), (2048, 2)])
def test_batch_tiles_agree_with_the_default_shape(threads, tile):
    """Every launch shape the autotuner may pick (threads per scene x contacts in flight per
    thread; 2048 = a cluster of two CTAs per scene) solves the same problems: positions
    within 1e-9 of the default 256 x 4 shape."""
    scenes = small_piles(5, 100, 1500, seed=10)
    ref = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, block_threads=256, tile=4, **KW).run(ST["dt"], 4)
    b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, block_threads=threads, tile=tile, **KW).run(ST["dt"], 4)
    assert b.block_threads() == threads and b.tile() == tile
    for s in range(len(scenes)):
        assert rel_err(b.scene(s).pos, ref.scene(s).pos) <= 1e-9, s
    with pytest.raises(ScopiGPUError):
        ScopiBatch(scenes, vap=ST["vap"], block_threads=256, tile=1, **KW)


def test_batch_autotune_graph_replay_and_launch_count():
    scenes = small_piles(8, 100, 1500, seed=11)
    b = ScopiBatch(scenes, vap=ST["vap"], precision=MIXED, **KW)
    b.run(ST["dt"], 1)
    assert b.block_threads() in (256, 512, 1024, 2048) and b.tile() in (1, 2, 4)
    b.run(ST["dt"], 1)  # captures the graph, replays it once
    l1 = b.kernel_launches()
    b.run(ST["dt"], 1)
    l2 = b.kernel_launches()
    b.run(ST["dt"], 3)
    l3 = b.kernel_launches()
    per_step = l2 - l1
    assert per_step > 0 and l3 - l2 == 3 * per_step
    assert b.stats()["steps"] == 6
    with pytest.raises(ScopiGPUError):
        b._check(b._lib.scopi_gpu_batch_set_block_threads(b._h, 512), "set_block_threads")


def test_batch_rejects_bad_block_size_and_viscous_friction():
    scenes = small_piles(2)
    with pytest.raises(ScopiGPUError):
        ScopiBatch(scenes, block_threads=300, **KW)
    b = ScopiBatch(scenes, **KW)
    assert b._lib.scopi_gpu_batch_set_block_threads(b._h, 512) == 0
    # 2048 = the cluster shape with its default tile
    assert b._lib.scopi_gpu_batch_set_block_threads(b._h, 2048) == 0
    assert b._lib.scopi_gpu_batch_set_block_threads(b._h, 4096) < 0
    b.run(ST["dt"], 1)
    assert b.block_threads() == 2048 and b.tile() == 1
    from scopi_b200 import VISCOUS_FRICTION
    with pytest.raises(ScopiGPUError):
        ScopiBatch(scenes, problem=VISCOUS_FRICTION, **KW)


def test_batch_cluster_shape_mixed_meets_violation_target():
    """The mixed form with two CTAs per scene (its FP64 residual and corrections included)
    keeps every step's violation at or below 1e-6."""
    scenes = small_piles(4, 200, 2000, seed=13)
    b = ScopiBatch(scenes, vap=ST["vap"], precision=MIXED, block_threads=2048, tile=1, mixed_violation_tol=1e-6,
                   **KW)
    for _ in range(10):
        b.run(ST["dt"], 1)
        st = b.stats()
        assert st["violation"] <= 1e-6 and st["converged"] == 1, st
    assert b.block_threads() == 2048
    b.close()


def test_batch_autotune_waits_for_a_nontrivial_step():
    """Falling piles converge in one iteration for their first steps: no tuning on those."""
    scenes = configs.pile_scenes(4, seed=12, nmin=50, nmax=200)
    b = ScopiBatch(scenes, vap=ST["vap"], precision=MIXED, **KW).run(ST["dt"], 2)
    assert max(b.scene_stats(s)["iterations"] for s in range(4)) < 64
    assert b.block_threads() == 512


def test_batch_mixed_keeps_violation_target_through_landing():
    """Disks landing on the segment: the reference's fixed first step alpha = 0.05 can stop
    a solve after one iteration with a resting contact still open by ~ g dt^2 (the FP64
    drop-in reproduces that); the mixed form's curvature start keeps every step <= 1e-6."""
    scenes = configs.pile_scenes(12, seed=13, nmin=200, nmax=1000)
    b = ScopiBatch(scenes, vap=ST["vap"], precision=MIXED, mixed_violation_tol=1e-6, **KW)
    worst = 0.0
    for _ in range(70):
        b.run(ST["dt"], 1)
        worst = max(worst, b.stats()["violation"])
    assert worst <= 1e-6


# ---- Friction scenes (LagrangeMultiplier<Friction>, lagrange_multiplier.hpp:208-273): the
# 6-dof rows solved per scene in FP64, one CTA per scene (k_apgd_batch6)
FKW = dict(KW, mu=0.3)


def test_batch_friction_matches_oracle_per_scene():
    scenes = small_piles(4)
    steps = 8
    b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, problem=FRICTION, **FKW)
    oracles = [oracle_solver(s, vap=ST["vap"], problem=FRICTION, **FKW) for s in scenes]
    for k in range(steps):
        b.run(ST["dt"], 1)
        for s, o in enumerate(oracles):
            o.run(ST["dt"], 1)
            assert b.scene_stats(s)["contacts"] == len(o.contacts()["i"]), f"scene {s} step {k}"
    iters = 0
    for s, o in enumerate(oracles):
        g = b.scene(s)
        st = b.scene_stats(s)
        print(s, "positions", rel_err(g.pos, o.pa.pos), "velocities", rel_err(g.v, o.pa.v),
              "omega", rel_err(g.omega, o.pa.omega), st)
        assert rel_err(g.pos, o.pa.pos) <= 1e-9, s
        assert rel_err(g.v, o.pa.v) <= 1e-7, s
        assert rel_err(g.omega, o.pa.omega) <= 1e-6, s
        assert st["converged"] == 1
        iters = max(iters, st["iterations"])
    assert iters > 10
    b.close()


def test_batch_friction_matches_single_scene_gpu():
    scenes = small_piles(5, 100, 800, seed=9) + [lone_disk()]
    steps = 5
    b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, problem=FRICTION, **FKW).run(ST["dt"], steps)
    for s, pa in enumerate(scenes):
        one = ScopiSolver(pa, vap=ST["vap"], precision=FP64, problem=FRICTION, **FKW).run(ST["dt"], steps)
        g = b.scene(s)
        assert b.scene_stats(s)["contacts"] == one.stats()["contacts"], s
        assert rel_err(g.pos, one.particles.pos) <= 1e-9, s
        assert rel_err(g.v, one.particles.v) <= 1e-7, s
        assert b.scene_stats(s)["violation"] <= 1e-5, (s, b.scene_stats(s))
        one.close()
    b.close()


def test_batch_friction_refuses_mixed_precision():
    with pytest.raises(ScopiGPUError):
        ScopiBatch(small_piles(2), vap=ST["vap"], precision=MIXED, problem=FRICTION, **FKW)


# ---- Viscous scenes (LagrangeMultiplier<Viscous>, lagrange_multiplier.hpp:116-206; gamma
# carried by (i, j) from step to step, solver.hpp:241-258): FP64, one CTA per scene
def test_batch_viscous_matches_oracle_per_scene():
    from scopi_b200 import VISCOUS
    scenes = small_piles(4)
    steps = 10
    b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, problem=VISCOUS, **KW)
    oracles = [oracle_solver(s, vap=ST["vap"], problem=VISCOUS, **KW) for s in scenes]
    for k in range(steps):
        b.run(ST["dt"], 1)
        for s, o in enumerate(oracles):
            o.run(ST["dt"], 1)
            assert b.scene_stats(s)["contacts"] == len(o.contacts()["i"]), f"scene {s} step {k}"
    for s, o in enumerate(oracles):
        g = b.scene(s)
        st = b.scene_stats(s)
        print(s, "positions", rel_err(g.pos, o.pa.pos), "velocities", rel_err(g.v, o.pa.v), st)
        assert rel_err(g.pos, o.pa.pos) <= 1e-9, s
        assert rel_err(g.v, o.pa.v) <= 1e-7, s
        assert st["converged"] == 1
    b.close()


def test_batch_viscous_matches_single_scene_gpu():
    from scopi_b200 import VISCOUS
    scenes = small_piles(5, 100, 800, seed=14) + [lone_disk()]
    steps = 8
    b = ScopiBatch(scenes, vap=ST["vap"], precision=FP64, problem=VISCOUS, **KW).run(ST["dt"], steps)
    for s, pa in enumerate(scenes):
        one = ScopiSolver(pa, vap=ST["vap"], precision=FP64, problem=VISCOUS, **KW).run(ST["dt"], steps)
        g = b.scene(s)
        assert b.scene_stats(s)["contacts"] == one.stats()["contacts"], s
        assert rel_err(g.pos, one.particles.pos) <= 1e-9, s
        assert rel_err(g.v, one.particles.v) <= 1e-7, s
        one.close()
    b.close()
