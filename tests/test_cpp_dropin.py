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
@pytest.mark.parametrize("mode,name", [("nofriction", "3spheres_nofriction"), ("viscous", "3spheres_viscous"),
                                       ("viscous_friction", "3spheres_viscous_friction")])
def test_cpp_api_matches_reference_golden(exe, golden, mode, name, tmp_path):
    res = json.loads(subprocess.run([exe, mode], check=True, capture_output=True, text=True, cwd=tmp_path).stdout)
    worst = 0.0
    for got, ref in zip(res["objects"], golden[name]["objects"]):
        for key in ("position", "velocity", "omega", "quaternion"):
            for a, b in zip(got[key], ref[key]):
                worst = max(worst, abs(a - b))
    assert worst <= 1e-5, worst


WORM_SRC = os.path.join(ROOT, "tests", "cpp", "two_worms_dropin.cpp")
PER_SRC = os.path.join(ROOT, "tests", "cpp", "periodic_dropin.cpp")
SE_SRC = os.path.join(ROOT, "tests", "cpp", "superellipsoids_dropin.cpp")
SE2_SRC = os.path.join(ROOT, "tests", "cpp", "two_ellipsoids_dropin.cpp")
FP_SRC = os.path.join(ROOT, "tests", "cpp", "fixed_point_dropin.cpp")
RS_SRC = os.path.join(ROOT, "tests", "cpp", "restart_dropin.cpp")


@pytest.mark.parametrize("src", [SE_SRC, SE2_SRC, FP_SRC, RS_SRC, WORM_SRC, PER_SRC])
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
def test_cpp_two_ellipsoids_match_reference_golden(se2_exe, golden, mode, tol, tmp_path):
    """test/test_superellipsoid.cpp:451-581 through the C++ API against two_ellipsoids_*.json."""
    res = json.loads(subprocess.run([se2_exe, mode], check=True, capture_output=True, text=True, cwd=tmp_path).stdout)
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
    res = json.loads(subprocess.run([se_exe, scene], check=True, capture_output=True, text=True, cwd=tmp_path).stdout)
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
def test_cpp_friction_fixed_point_matches_analytic(fp_exe, tmp_path):
    """test/test_gradient.cpp:215-283 through the C++ API: errors against the analytic rolling
    solution within the reference's bounds (pos, q 1e-2; v, omega 1e-12 under doctest::Approx)."""
    import math

    import scenes as S
    res = json.loads(subprocess.run([fp_exe], check=True, capture_output=True, text=True, cwd=tmp_path).stdout)
    x, theta, v, om = S.analytic_friction(math.pi / 4, 0.5, 0.01 * 500, 1.0, 1.0, 2.0)
    qa = S.quaternion(theta)
    e_pos = math.hypot(res["position"][0] - x[0], res["position"][1] - x[1]) / math.hypot(*x)
    e_q = math.sqrt(sum((a - b) ** 2 for a, b in zip(res["quaternion"], qa))) / math.sqrt(sum(b * b for b in qa))
    e_v = math.hypot(res["velocity"][0] - v[0], res["velocity"][1] - v[1]) / math.hypot(*v)
    e_om = (res["omega"] - om) ** 2 / om ** 2
    assert e_pos <= 1e-2 and e_q <= 1e-2, (e_pos, e_q)
    assert e_v <= 1.2e-5 and e_om <= 1.2e-5, (e_v, e_om)


# ------------------------------------------------------------------ snapshot files
SNAP_SRC = os.path.join(ROOT, "tests", "cpp", "snapshot_writer.cpp")
SNAPSHOT_FIXTURE = os.path.join(ROOT, "tests", "golden", "snapshot_obstacles_sphere_sphere_moving.json")
WORM_FIXTURE = os.path.join(ROOT, "tests", "golden", "snapshot_two_worms.json")
# keys of write_objects.hpp per shape and of the properties written by solver.hpp:383-400
OBJECT_KEYS = {
    "sphere": {"id", "position", "properties", "quaternion", "radius", "rotation", "type"},
    "plane": {"id", "normal", "position", "properties", "quaternion", "rotation", "type"},
    "segment": {"id", "normal", "p1", "p2", "properties", "quaternion", "tangent", "type"},
    "superellipsoid": {"id", "position", "properties", "quaternion", "radius", "rotation", "squareness", "type"},
}
PROPERTY_KEYS = {"active", "desired_omega", "desired_velocity", "force", "mass", "moment_inertia", "omega", "velocity"}


def bson_decode(b, pos=0, array=False):
    """Minimal BSON reader (the element types the writer emits)."""
    import struct
    n = struct.unpack_from("<i", b, pos)[0]
    end, pos = pos + n - 1, pos + 4
    out = {}
    while pos < end:
        t = b[pos]
        k = b.index(b"\0", pos + 1)
        key, pos = b[pos + 1:k].decode(), k + 1
        if t == 0x01:
            v, pos = struct.unpack_from("<d", b, pos)[0], pos + 8
        elif t == 0x02:
            ln = struct.unpack_from("<i", b, pos)[0]
            v, pos = b[pos + 4:pos + 4 + ln - 1].decode(), pos + 4 + ln
        elif t in (0x03, 0x04):
            ln = struct.unpack_from("<i", b, pos)[0]
            v, pos = bson_decode(b, pos, t == 0x04), pos + ln
        elif t == 0x08:
            v, pos = bool(b[pos]), pos + 1
        elif t == 0x0A:
            v = None
        elif t == 0x10:
            v, pos = struct.unpack_from("<i", b, pos)[0], pos + 4
        elif t == 0x12:
            v, pos = struct.unpack_from("<q", b, pos)[0], pos + 8
        else:
            raise ValueError(f"BSON type {t:#x}")
        out[key] = v
    return [out[str(i)] for i in range(len(out))] if array else out


def test_snapshot_writer_formats(tmp_path):
    """write_output_files' documents for every shape (2D and 3D): the reference's fields per
    object, the values of the container, and the same document in BSON."""
    import math
    exe = str(tmp_path / "snapw")
    subprocess.run([GXX, "-std=c++17", "-Wall", "-Werror", *INC, SNAP_SRC, "-o", exe], check=True)
    subprocess.run([exe, str(tmp_path), SNAPSHOT_FIXTURE], check=True)
    for name in ("snap2d", "snap3d"):
        with open(tmp_path / f"{name}.json") as fh:
            doc = json.load(fh)
        with open(tmp_path / f"{name}.bson", "rb") as fh:
            assert bson_decode(fh.read()) == doc
        assert doc["contacts"] is None
        for o in doc["objects"]:
            assert set(o) == OBJECT_KEYS[o["type"]], o["type"]
            assert set(o["properties"]) == PROPERTY_KEYS
    d2 = json.load(open(tmp_path / "snap2d.json"))["objects"]
    assert [o["type"] for o in d2] == ["plane", "segment", "sphere", "superellipsoid"]
    assert [o["properties"]["active"] for o in d2] == [False, False, True, True]
    # plane(pi/3): normal = column 0 of R; segment: the given extrema, tangent = (-n1, n0)
    assert abs(d2[0]["normal"][0] - 0.5) < 1e-15 and abs(d2[0]["normal"][1] - math.sqrt(3) / 2) < 1e-15
    assert max(abs(a - b) for a, b in zip(d2[1]["p1"] + d2[1]["p2"], [-1.0, 0.5, 2.0, 1.5])) < 1e-14
    assert d2[1]["tangent"] == [-d2[1]["normal"][1], d2[1]["normal"][0]]
    s = d2[2]
    assert s["position"] == [0.3, 1.2] and s["radius"] == 0.25
    assert s["properties"]["velocity"] == [1.0, -2.0] and s["properties"]["mass"] == 2.0
    assert s["properties"]["moment_inertia"] == 0.3 and s["properties"]["force"] == [0.0, -9.81]
    assert d2[3]["radius"] == [0.2, 0.1] and d2[3]["squareness"] == [1.2] and d2[3]["properties"]["omega"] == 0.5
    d3 = json.load(open(tmp_path / "snap3d.json"))["objects"]
    assert d3[0]["properties"]["moment_inertia"] == [0.1, 0.2, 0.3] and d3[0]["properties"]["omega"] == [1.0, 2.0, 3.0]
    assert d3[1]["radius"] == [0.3, 0.2, 0.1] and d3[1]["squareness"] == [0.8, 1.3]
    assert len(d3[1]["rotation"]) == 9


@pytest.mark.gpu
@pytest.mark.parametrize("mode,name", [("nofriction", "3spheres_nofriction"), ("viscous", "3spheres_viscous"),
                                       ("viscous_friction", "3spheres_viscous_friction")])
def test_cpp_snapshot_files_match_reference_golden(exe, golden, mode, name, tmp_path):
    """The reference's "3 Spheres" tests with snapshot files (output_frequency = total_it):
    the initial snapshot and the final one, whose objects agree with the reference's golden
    file as its diffFile checks them (test/utils.cpp:14-75, numbers within 1e-5)."""
    subprocess.run([exe, mode, str(tmp_path / "out")], check=True, capture_output=True, cwd=tmp_path)
    total = 60 if mode == "nofriction" else 70
    first = json.load(open(tmp_path / "out" / f"{name}_0000.json"))
    last = json.load(open(tmp_path / "out" / f"{name}_{total:04d}.json"))
    assert sorted(os.listdir(tmp_path / "out")) == [f"{name}_0000.json", f"{name}_{total:04d}.json"]
    assert first["contacts"] is None and [o["position"] for o in first["objects"]] == [
        [-1.7, 1.3], [0.5, 1.7], [4.5, 1.3]]
    worst = 0.0
    for got, ref in zip(last["objects"], golden[name]["objects"]):
        assert set(got) == OBJECT_KEYS["sphere"] and set(got["properties"]) == PROPERTY_KEYS
        assert got["type"] == ref["type"] and got["properties"]["active"] == ref["active"]
        for key in ("position", "quaternion"):
            worst = max(worst, max(abs(a - b) for a, b in zip(got[key], ref[key])))
        worst = max(worst, max(abs(a - b) for a, b in zip(got["properties"]["velocity"], ref["velocity"])))
        worst = max(worst, abs(got["properties"]["omega"] - ref["omega"][0]))
    assert worst <= 1e-5, worst


def test_restart_reads_snapshots(tmp_path):
    """from_json (restart.hpp:20-67): the writer's own files read back and written again give
    the same document (numbers to 1e-12: a segment is rebuilt from its extrema, which moves
    them by an ulp, as in the reference), and two snapshots the reference wrote (test/references/
    obstacles_sphere_sphere_moving.json, two_worms.json) give back every object and property
    they hold."""
    exe = str(tmp_path / "snapw")
    subprocess.run([GXX, "-std=c++17", "-Wall", "-Werror", *INC, SNAP_SRC, "-o", exe], check=True)
    subprocess.run([exe, str(tmp_path), SNAPSHOT_FIXTURE, WORM_FIXTURE], check=True)
    def close(a, b):
        if isinstance(a, dict):
            return isinstance(b, dict) and a.keys() == b.keys() and all(close(a[k], b[k]) for k in a)
        if isinstance(a, list):
            return isinstance(b, list) and len(a) == len(b) and all(close(x, y) for x, y in zip(a, b))
        if isinstance(a, float):
            return isinstance(b, float) and abs(a - b) <= 1e-12
        return a == b

    for name in ("snap2d", "snap3d"):
        assert close(json.load(open(tmp_path / f"{name}.json")), json.load(open(tmp_path / f"{name}_rt.json")))
    ref = json.load(open(SNAPSHOT_FIXTURE))["objects"]
    got = json.load(open(tmp_path / "snapfile_rt.json"))["objects"]
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        for key in ("type", "id", "position", "quaternion", "radius", "rotation", "properties"):
            assert g[key] == r[key], (key, g[key], r[key])
    # worms (restart.hpp:53-64, write_objects.hpp:183-198): two objects of six spheres each
    ref = json.load(open(WORM_FIXTURE))["objects"]
    got = json.load(open(tmp_path / "wormfile_rt.json"))["objects"]
    assert len(got) == len(ref) == 2
    for g, r in zip(got, ref):
        assert g.keys() == r.keys() and g["type"] == "worm"
        assert g["worm"] == r["worm"] and g["properties"] == r["properties"]


@pytest.mark.gpu
def test_cpp_restart_continues_like_one_run(tmp_path):
    """30 steps, a snapshot, from_json and 30 more steps with a new solver end in the state
    of 60 steps in one run, bit for bit (NoFriction carries nothing else between steps, and
    the snapshot's numbers read back exactly)."""
    from scopi_b200 import build
    build.build()
    exe = str(tmp_path / "restart")
    lib = os.path.join(ROOT, "scopi_b200")
    subprocess.run([GXX, "-O2", "-std=c++17", *INC, RS_SRC, "-L", lib, "-lscopi_gpu", f"-Wl,-rpath,{lib}", "-o", exe],
                   check=True)
    one = json.loads(subprocess.run([exe], check=True, capture_output=True, text=True, cwd=tmp_path).stdout)
    two = json.loads(subprocess.run([exe, "restart", str(tmp_path / "snap")], check=True, capture_output=True,
                                    text=True, cwd=tmp_path).stdout)
    assert os.path.exists(tmp_path / "snap" / "restart_0030.json")
    assert one == two


def diff_file(result, ref, tol):
    """test/utils.cpp:14-75 (diffFile): the "objects" of the two documents may differ only in
    floating-point entries, each by at most tol."""
    def walk(a, b, path):
        if isinstance(b, float) and isinstance(a, float):
            assert abs(a - b) <= tol, (path, a, b)
        elif isinstance(b, dict):
            assert isinstance(a, dict) and a.keys() == b.keys(), path
            for k in b:
                walk(a[k], b[k], path + "/" + k)
        elif isinstance(b, list):
            assert isinstance(a, list) and len(a) == len(b), path
            for k, (x, y) in enumerate(zip(a, b)):
                walk(x, y, f"{path}/{k}")
        else:
            assert a == b and type(a) is type(b), (path, a, b)
    walk(result["objects"], ref["objects"], "")


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["kdtree", "brute_force"])
def test_cpp_two_worms_match_reference_golden(method, tmp_path):
    """The reference's "two worms" test (test/test_worm.cpp:480-530, both contact methods)
    through the C++ drop-in: its final snapshot file passes the reference's own golden-file
    check against test/references/two_worms.json (tolerance 1e-6), and its contact list is the
    reference's (pairs, and the glued links after the sorted list)."""
    exe = str(tmp_path / "worms")
    lib = os.path.join(ROOT, "scopi_b200")
    subprocess.run([GXX, "-O2", "-std=c++17", *INC, WORM_SRC, "-L", lib, "-lscopi_gpu", f"-Wl,-rpath,{lib}", "-o", exe],
                   check=True)
    subprocess.run([exe, method, str(tmp_path / "out")], check=True, capture_output=True, cwd=tmp_path)
    got = json.load(open(tmp_path / "out" / "two_worms_1000.json"))
    ref = json.load(open(WORM_FIXTURE))
    diff_file(got, ref, 1e-6)
    assert [(c["i"], c["j"]) for c in got["contacts"]] == [(c["i"], c["j"]) for c in ref["contacts"]]
    for g, r in zip(got["contacts"], ref["contacts"]):
        assert abs(g["distance"] - r["distance"]) <= 1e-6
        assert max(abs(a - b) for a, b in zip(g["normal"], r["normal"])) <= 1e-6


@pytest.mark.gpu
def test_cpp_periodic_box_matches_oracle(tmp_path):
    """ScopiSolver(BoxDomain, particles) through the C++ drop-in: the two disks meeting across
    the periodic bound end where the oracle's do."""
    import scenes as S
    from gpu_helpers import oracle_solver
    exe = str(tmp_path / "periodic")
    lib = os.path.join(ROOT, "scopi_b200")
    subprocess.run([GXX, "-O2", "-std=c++17", *INC, PER_SRC, "-L", lib, "-lscopi_gpu", f"-Wl,-rpath,{lib}", "-o", exe],
                   check=True)
    res = json.loads(subprocess.run([exe], check=True, capture_output=True, text=True, cwd=tmp_path).stdout)
    pa, kw, dt, total = S.periodic_two_disks()
    o = oracle_solver(pa, **kw).run(dt, total)
    for k in range(2):
        for d in range(2):
            assert abs(res["positions"][k][d] - o.pa.pos[k, d]) <= 1e-8
    assert res["contacts"] == 1


def test_worm_container_like_reference(tmp_path):
    """test/test_worm.cpp:26-478 (construction and indexing of 2D and 3D worms, alone and in a
    container) on the drop-in's worm<dim> and scopi_container, without a GPU."""
    exe = str(tmp_path / "wormc")
    src = os.path.join(ROOT, "tests", "cpp", "worm_container.cpp")
    subprocess.run([GXX, "-std=c++17", "-Wall", "-Werror", *INC, src, "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_box_domain_api(tmp_path):
    """BoxDomain<dim> (box.hpp): corners, periodic axes and accessors, without a GPU."""
    exe = str(tmp_path / "box")
    src = os.path.join(ROOT, "tests", "cpp", "box_domain.cpp")
    subprocess.run([GXX, "-std=c++17", "-Wall", "-Werror", *INC, src, "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


CM_SRC = os.path.join(ROOT, "tests", "cpp", "contacts_matrices_dropin.cpp")


def test_contacts_matrices_header_compiles():
    subprocess.run([GXX, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", *INC, CM_SRC], check=True)


@pytest.mark.gpu
def test_cpp_contact_methods_and_matrices(tmp_path):
    """contact_kdtree(params).run(particles), contact_brute_force, AMatrix / ATMatrix as the
    reference's test_contacts_kdtree.cpp, test_contacts_brute_force.cpp and test_matrices.cpp
    use them."""
    from scopi_b200 import build
    build.build()
    out = str(tmp_path / "contacts_matrices")
    lib = os.path.join(ROOT, "scopi_b200")
    subprocess.run([GXX, "-O2", "-std=c++17", *INC, CM_SRC, "-L", lib, "-lscopi_gpu", f"-Wl,-rpath,{lib}", "-o", out],
                   check=True)
    r = subprocess.run([out], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout)
    assert res["failures"] == 0
    assert abs(res["adjoint_difference"]) <= 1e-12
