"""Extract the golden end states of the reference's solver regression tests.

Reads the reference's own golden snapshots (test/references/*.json of
hpc-maths/scopi, written by ScopiSolver::write_output_files) and keeps only what
the parity tests compare: per object position, quaternion, velocity and omega
(the fields test/utils.cpp:14-75 diffs; for a worm the position and quaternion of
each of its spheres), plus the contact list of the last
step (i, j, distance, normal, pi, pj).  Writes tests/golden/reference_states.json, and
two snapshot files unchanged (snapshot_obstacles_sphere_sphere_moving.json,
snapshot_two_worms.json) for the restart tests.

Run once in a checkout that has the reference at REF (default /root/reference):
    python tests/golden/make_golden.py [REF]
"""
import json
import os
import sys

FILES = [
    "3spheres_nofriction",          # test/test_gradient.cpp:377-439
    "3spheres_viscous",             # test/test_gradient.cpp:441-503
    "3spheres_friction_fp",         # test/test_gradient.cpp:505-572 (FrictionFixedPoint)
    "3spheres_viscous_friction",    # test/test_gradient.cpp:574-642 (ViscousFriction)
    "sphere_plane_friction_mu01",   # test/test_gradient.cpp:156-213
    "two_spheres_asymmetrical",     # test/test_sphere.cpp:341-380
    "two_spheres_symmetrical",      # test/test_sphere.cpp:382-421
    "2d_case_spheres",              # test/test_sphere.cpp:423-484
    "obstacles_sphere_sphere_moving",  # test/test_obstacles.cpp:214-250
    "two_worms",                    # test/test_worm.cpp:480-530
    # Friction with vap_fixed (test/test_friction.cpp, which the reference's test build leaves
    # out); older output format, written before the motion of their step
    "two_spheres_asymmetrical_friction",  # test/test_friction.cpp:17-53
    "2d_case_spheres_friction",           # test/test_friction.cpp:55-112
    # superellipsoids (2D); these snapshots use an older output format (no velocities,
    # contacts without i, j and distance), written before the motion of their step
    "two_ellipsoids_symmetrical",           # test/test_superellipsoid.cpp:451-491
    "two_ellipsoids_spheres_symmetrical",   # test/test_superellipsoid.cpp:493-536
    "two_ellipsoids_asymmetrical",          # test/test_superellipsoid.cpp:538-581
    "two_ellipsoids_spheres_asymmetrical",  # test/test_superellipsoid.cpp:583-628
    "2d_case_superellipsoid",               # test/test_superellipsoid.cpp:630-702
]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    out = {}
    for name in FILES:
        with open(os.path.join(ref, "test", "references", name + ".json")) as fh:
            d = json.load(fh)
        objs = []
        for o in d["objects"]:
            if "properties" not in o:  # older format: geometry only
                objs.append({"type": o["type"], "position": o["position"], "quaternion": o["quaternion"],
                             "radius": o["radius"], "squareness": o.get("squareness")})
                continue
            p = o["properties"]
            om = p["omega"]
            if o["type"] == "worm":  # one object, one sphere per body; properties of its first body
                objs.append({
                    "type": "worm",
                    "active": p["active"],
                    "spheres": [{"id": w["id"], "position": w["position"], "quaternion": w["quaternion"],
                                 "radius": w["radius"]} for w in o["worm"]],
                    "velocity": p["velocity"],
                    "omega": om if isinstance(om, list) else [om],
                })
                continue
            objs.append({
                "type": o["type"],
                "active": p["active"],
                "position": o["position"],
                "quaternion": o["quaternion"],
                "velocity": p["velocity"],
                "omega": om if isinstance(om, list) else [om],
            })
        contacts = []
        for c in d.get("contacts") or []:
            if "nij" in c:  # older format
                contacts.append({"normal": c["nij"], "pi": c["pi"], "pj": c["pj"]})
            else:
                contacts.append({k: c[k] for k in ("i", "j", "distance", "normal", "pi", "pj")})
        out[name] = {"objects": objs, "contacts": contacts}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_states.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", dst)
    # two snapshots kept whole, as the reference wrote them: the inputs of the restart tests
    # (from_json, restart.hpp:20-67)
    for name in ("obstacles_sphere_sphere_moving", "two_worms"):
        src = os.path.join(ref, "test", "references", name + ".json")
        dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "snapshot_" + name + ".json")
        with open(src) as fh, open(dst, "w") as out_fh:
            out_fh.write(fh.read())
        print("wrote", dst)


if __name__ == "__main__":
    main()
