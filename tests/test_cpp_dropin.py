"""The C++ scopi:: API (scopi_b200/include) used exactly like the reference's own tests.

CPU: the headers compile (reference-style scene code, the demo with GPU policy types).
GPU: the reference's "3 Spheres" scenes run through the C++ API and the C ABI and
match the reference's golden snapshots (test/test_gradient.cpp:377-503, tol 1e-5).
"""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
INC = ["-I", os.path.join(ROOT, "scopi_b200", "include"), "-I", os.path.join(ROOT, "include")]
SRC = os.path.join(ROOT, "tests", "cpp", "three_spheres_dropin.cpp")
DEMO = os.path.join(ROOT, "scopi_b200", "demos", "box_spheres_3d.cpp")


@pytest.mark.parametrize("src", [SRC, DEMO])
def test_headers_compile(src):
    subprocess.run([GXX, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", *INC, src], check=True)


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    from scopi_b200 import build
    build.build()
    out = str(tmp_path_factory.mktemp("cpp") / "three_spheres")
    lib = os.path.join(ROOT, "scopi_b200")
    subprocess.run([GXX, "-O2", "-std=c++17", *INC, SRC, "-L", lib, "-lscopi_gpu", f"-Wl,-rpath,{lib}", "-o", out],
                   check=True)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("mode,name", [("nofriction", "3spheres_nofriction"), ("viscous", "3spheres_viscous")])
def test_cpp_api_matches_reference_golden(exe, golden, mode, name):
    res = json.loads(subprocess.run([exe, mode], check=True, capture_output=True, text=True).stdout)
    worst = 0.0
    for got, ref in zip(res["objects"], golden[name]["objects"]):
        for key in ("position", "velocity", "omega", "quaternion"):
            for a, b in zip(got[key], ref[key]):
                worst = max(worst, abs(a - b))
    assert worst <= 1e-5, worst


SE_SRC = os.path.join(ROOT, "tests", "cpp", "superellipsoids_dropin.cpp")
SE2_SRC = os.path.join(ROOT, "tests", "cpp", "two_ellipsoids_dropin.cpp")
FP_SRC = os.path.join(ROOT, "tests", "cpp", "fixed_point_dropin.cpp")


@pytest.mark.parametrize("src", [SE_SRC, SE2_SRC, FP_SRC])
def test_superellipsoid_header_compiles(src):
    subprocess.run([GXX, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", *INC, src], check=True)


@pytest.fixture(scope="module")
def se2_exe(tmp_path_factory):
    from scopi_b200 import build
    build.build()
    out = str(tmp_path_factory.mktemp("cpp") / "two_ellipsoids")
    lib = os.path.join(ROOT, "scopi_b200")
    subprocess.run([GXX, "-O2", "-std=c++17", *INC, SE2_SRC, "-L", lib, "-lscopi_gpu", f"-Wl,-rpath,{lib}", "-o", out],
                   check=True)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("mode,tol", [("symmetrical", 1e-6), ("asymmetrical", 5e-6)])
def test_cpp_two_ellipsoids_match_reference_golden(se2_exe, golden, mode, tol):
    """test/test_superellipsoid.cpp:451-581 through the C++ API against two_ellipsoids_*.json."""
    res = json.loads(subprocess.run([se2_exe, mode], check=True, capture_output=True, text=True).stdout)
    gold = golden["two_ellipsoids_" + mode]
    worst = 0.0
    for got, ref in zip(res["objects"], gold["objects"]):
        for key in ("position", "quaternion"):
            worst = max(worst, max(abs(a - b) for a, b in zip(got[key], ref[key])))
    assert len(res["contacts"]) == len(gold["contacts"])
    for got, ref in zip(res["contacts"], gold["contacts"]):
        worst = max(worst, max(abs(a - b) for a, b in zip(got["nij"], ref["normal"])))
        for key in ("pi", "pj"):
            worst = max(worst, max(abs(a - b) for a, b in zip(got[key], ref[key])))
    assert worst <= tol, worst


@pytest.fixture(scope="module")
def se_exe(tmp_path_factory):
    from scopi_b200 import build
    build.build()
    out = str(tmp_path_factory.mktemp("cpp") / "superellipsoids")
    lib = os.path.join(ROOT, "scopi_b200")
    subprocess.run([GXX, "-O2", "-std=c++17", *INC, SE_SRC, "-L", lib, "-lscopi_gpu", f"-Wl,-rpath,{lib}", "-o", out],
                   check=True)
    return out


def write_scene(path, pa, steps, dt, mu, dmax, kd, tol, max_ite):
    with open(path, "w") as fh:
        fh.write(f"{len(pa.shape)} {steps} {dt!r} {mu!r} {dmax!r} {kd!r} {tol!r} {max_ite}\n")
        for b in range(len(pa.shape)):
            vals = [int(pa.shape[b]), int(b >= pa.nb_inactive), *pa.pos[b], *pa.q[b], *pa.axes[b],
                    *pa.squareness[b], pa.m[b], *pa.j[b], *pa.f[b], *pa.v[b]]
            fh.write(" ".join(repr(float(x)) if not isinstance(x, int) else str(x) for x in vals) + "\n")


@pytest.mark.gpu
def test_cpp_superellipsoid_pile_matches_python_api_and_oracle(se_exe, tmp_path):
    """The same pile through the C++ API, the Python API (same engine: bitwise equal) and
    the oracle (same contacts; positions to the bound of the superellipsoid parity tests)."""
    import numpy as np

    from gpu_helpers import gpu_solver, oracle_solver, rel_err
    from scopi_b200 import FRICTION, configs
    pa = configs.se_pile(count=27, side=3, seed=4)
    st = configs.SETTINGS["se_pile"]
    kd = configs.se_kd_radius(pa, st["dmax"])
    steps = 4
    scene = str(tmp_path / "scene.txt")
    write_scene(scene, pa, steps, st["dt"], st["mu"], st["dmax"], kd, st["tolerance"], st["max_ite"])
    res = json.loads(subprocess.run([se_exe, scene], check=True, capture_output=True, text=True).stdout)
    pos = np.array(res["positions"])
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"], mu=st["mu"],
              problem=FRICTION, kd_tree_radius=kd)
    g = gpu_solver(configs.se_pile(count=27, side=3, seed=4), **kw).run(st["dt"], steps)
    assert np.array_equal(pos, g.particles.pos)
    o = oracle_solver(configs.se_pile(count=27, side=3, seed=4), **kw).run(st["dt"], steps)
    oc = o.contacts()
    assert [tuple(c) for c in res["contacts"]] == list(zip(oc["i"].tolist(), oc["j"].tolist()))
    assert rel_err(pos, o.pa.pos) <= 2e-5


@pytest.fixture(scope="module")
def fp_exe(tmp_path_factory):
    from scopi_b200 import build
    build.build()
    out = str(tmp_path_factory.mktemp("cpp") / "fixed_point")
    lib = os.path.join(ROOT, "scopi_b200")
    subprocess.run([GXX, "-O2", "-std=c++17", *INC, FP_SRC, "-L", lib, "-lscopi_gpu", f"-Wl,-rpath,{lib}", "-o", out],
                   check=True)
    return out


@pytest.mark.gpu
def test_cpp_friction_fixed_point_matches_analytic(fp_exe):
    """test/test_gradient.cpp:215-283 through the C++ API: errors against the analytic rolling
    solution within the reference's bounds (pos, q 1e-2; v, omega 1e-12 under doctest::Approx)."""
    import math

    import scenes as S
    res = json.loads(subprocess.run([fp_exe], check=True, capture_output=True, text=True).stdout)
    x, theta, v, om = S.analytic_friction(math.pi / 4, 0.5, 0.01 * 500, 1.0, 1.0, 2.0)
    qa = S.quaternion(theta)
    e_pos = math.hypot(res["position"][0] - x[0], res["position"][1] - x[1]) / math.hypot(*x)
    e_q = math.sqrt(sum((a - b) ** 2 for a, b in zip(res["quaternion"], qa))) / math.sqrt(sum(b * b for b in qa))
    e_v = math.hypot(res["velocity"][0] - v[0], res["velocity"][1] - v[1]) / math.hypot(*v)
    e_om = (res["omega"] - om) ** 2 / om ** 2
    assert e_pos <= 1e-2 and e_q <= 1e-2, (e_pos, e_q)
    assert e_v <= 1.2e-5 and e_om <= 1.2e-5, (e_v, e_om)
