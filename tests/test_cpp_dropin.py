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
