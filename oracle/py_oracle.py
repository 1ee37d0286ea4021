"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
bench.py may import this module; the product package never does.  The oracle is
the C++17 restatement of the reference time step in scopi_oracle.cpp.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_scopi.so")

NOFRICTION, FRICTION, VISCOUS, FRICTION_FIXED_POINT, VISCOUS_FRICTION = 0, 1, 2, 3, 4
VAP_FIXED, VAP_FPD = 0, 1
BRUTE_FORCE, KDTREE = 0, 1


class OrcParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("problem", C.c_int32), ("vap", C.c_int32), ("contact_method", C.c_int32),
        ("dmax", C.c_double), ("kd_tree_radius", C.c_double), ("alpha", C.c_double), ("max_ite", C.c_int64),
        ("tolerance", C.c_double), ("dynamic_descent", C.c_int32), ("mu", C.c_double), ("gamma", C.c_double),
        ("gamma_min", C.c_double), ("gamma_tol", C.c_double), ("num_threads", C.c_int32),
        ("fixed_point_tol", C.c_double), ("fixed_point_max_iter", C.c_int64),
        ("box_lower", C.c_double * 3), ("box_upper", C.c_double * 3), ("periodic", C.c_int32 * 3),
    ]


class OrcParticles(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("nb_inactive", C.c_int64), ("shape", C.POINTER(C.c_int32)),
        ("pos", C.POINTER(C.c_double)), ("q", C.POINTER(C.c_double)), ("v", C.POINTER(C.c_double)),
        ("omega", C.POINTER(C.c_double)), ("vd", C.POINTER(C.c_double)), ("omega_d", C.POINTER(C.c_double)),
        ("f", C.POINTER(C.c_double)), ("m", C.POINTER(C.c_double)), ("j", C.POINTER(C.c_double)),
        ("radius", C.POINTER(C.c_double)), ("length", C.POINTER(C.c_double)),
        ("axes", C.POINTER(C.c_double)), ("squareness", C.POINTER(C.c_double)), ("worm", C.POINTER(C.c_int32)),
    ]


class OrcStats(C.Structure):
    _fields_ = [
        ("contacts", C.c_int64), ("iterations", C.c_int64), ("backtracks", C.c_int64), ("restarts", C.c_int64),
        ("converged", C.c_int32), ("violation", C.c_double), ("seconds_contacts", C.c_double),
        ("seconds_solve", C.c_double), ("seconds_other", C.c_double), ("fixed_point_iterations", C.c_int64),
    ]


_lib = None


def build() -> None:
    """Compile the oracle with its Makefile (g++, OpenMP, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcParticles)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_run.argtypes = [C.c_void_p, C.c_double, C.c_int64, C.c_int64]
        L.orc_get_particles.argtypes = [C.c_void_p, C.POINTER(OrcParticles)]
        L.orc_set_particles.argtypes = [C.c_void_p, C.POINTER(OrcParticles)]
        L.orc_num_contacts.restype = C.c_int64
        L.orc_num_contacts.argtypes = [C.c_void_p]
        P = C.POINTER(C.c_double)
        L.orc_get_contacts.restype = C.c_int64
        L.orc_get_contacts.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), P, P, P, P, P, C.c_int64]
        L.orc_get_lambda.restype = C.c_int64
        L.orc_get_lambda.argtypes = [C.c_void_p, P, C.c_int64]
        L.orc_get_stats.argtypes = [C.c_void_p, C.POINTER(OrcStats)]
        L.orc_detect.restype = C.c_int64
        L.orc_detect.argtypes = [C.c_void_p]
        L.orc_amat.argtypes = [C.c_void_p, P, P]
        L.orc_atmat.argtypes = [C.c_void_p, P, P]
        L.orc_se_se.restype = C.c_int
        L.orc_se_se.argtypes = [P, P, P]
        L.orc_se_plane.restype = C.c_int
        L.orc_se_plane.argtypes = [P, P, P]
        L.orc_se_se_system.argtypes = [P, P, P, P, P]
        L.orc_se_plane_residual.argtypes = [P, P, P, P]
        L.orc_se_se_hybrid.restype = C.c_int
        L.orc_se_se_hybrid.argtypes = [P, P, P, C.POINTER(C.c_int)]
        L.orc_se_se_from.restype = C.c_int
        L.orc_se_se_from.argtypes = [P, P, P, P]
        L.orc_se_se_start_value.restype = C.c_double
        L.orc_se_se_start_value.argtypes = [P, P, P]
        L.orc_se_se_start.restype = None
        L.orc_se_se_start.argtypes = [P, P, P]
        L.orc_se2_se2.restype = C.c_int
        L.orc_se2_se2.argtypes = [P, P, P]
        L.orc_se2_hybrid.restype = C.c_int
        L.orc_se2_hybrid.argtypes = [P, P, P, C.POINTER(C.c_int)]
        L.orc_se2_system.argtypes = [P, P, P, P, P]
        L.orc_sphere_se.restype = C.c_int
        L.orc_sphere_se.argtypes = [C.c_int, P, P, C.c_int, C.c_int, P]
        L.orc_se2_plane.restype = C.c_int
        L.orc_se2_plane.argtypes = [P, P, P]
        L.orc_lu_solve4.restype = C.c_int
        L.orc_lu_solve4.argtypes = [P, P, P]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _particles_struct(pa, keep):
    keep.append(pa)
    return OrcParticles(
        pa.n, pa.nb_inactive, pa.shape.ctypes.data_as(C.POINTER(C.c_int32)), _dp(pa.pos), _dp(pa.q), _dp(pa.v),
        _dp(pa.omega), _dp(pa.vd), _dp(pa.omega_d), _dp(pa.f), _dp(pa.m), _dp(pa.j), _dp(pa.radius), _dp(pa.length),
        _dp(pa.axes), _dp(pa.squareness), pa.worm.ctypes.data_as(C.POINTER(C.c_int32)),
    )


class OracleSolver:
    """Mirror of ``ScopiSolver<dim, problem, OptimGradient<apgd>, contact, vap>`` on the CPU."""

    def __init__(self, particles, problem=NOFRICTION, vap=VAP_FIXED, contact_method=KDTREE, dmax=2.0,
                 kd_tree_radius=17.0, alpha=0.05, max_ite=10000, tolerance=1e-7, dynamic_descent=True, mu=0.1,
                 gamma=0.0, gamma_min=-2.0, gamma_tol=1e-6, num_threads=0, fixed_point_tol=1e-6,
                 fixed_point_max_iter=1000, box_lower=(0.0, 0.0, 0.0), box_upper=(0.0, 0.0, 0.0), periodic=(0, 0, 0)):
        self.pa = particles.copy()
        self.params = OrcParams(particles.dim, problem, vap, contact_method, dmax, kd_tree_radius, alpha, max_ite,
                                tolerance, 1 if dynamic_descent else 0, mu, gamma, gamma_min, gamma_tol, num_threads,
                                fixed_point_tol, fixed_point_max_iter, (C.c_double * 3)(*box_lower),
                                (C.c_double * 3)(*box_upper), (C.c_int32 * 3)(*[int(bool(x)) for x in periodic]))
        keep = []
        ps = _particles_struct(self.pa, keep)
        self.h = lib().orc_create(C.byref(self.params), C.byref(ps))
        if not self.h:
            raise RuntimeError("orc_create failed")

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    def run(self, dt, total_it, initial_iter=0):
        rc = lib().orc_run(self.h, dt, total_it, initial_iter)
        if rc != 0:
            raise RuntimeError("orc_run failed")
        self.sync()
        return self

    def sync(self):
        keep = []
        ps = _particles_struct(self.pa, keep)
        lib().orc_get_particles(self.h, C.byref(ps))
        return self.pa

    def set_particles(self, pa):
        self.pa = pa.copy()
        keep = []
        ps = _particles_struct(self.pa, keep)
        lib().orc_set_particles(self.h, C.byref(ps))

    def detect(self):
        lib().orc_detect(self.h)
        return self.contacts()

    def contacts(self):
        n = lib().orc_num_contacts(self.h)
        ci = np.zeros(n, np.int64)
        cj = np.zeros(n, np.int64)
        d = np.zeros(n)
        g = np.zeros(n)
        nij = np.zeros((n, 3))
        pi = np.zeros((n, 3))
        pj = np.zeros((n, 3))
        lib().orc_get_contacts(self.h, ci.ctypes.data_as(C.POINTER(C.c_int64)), cj.ctypes.data_as(C.POINTER(C.c_int64)),
                               _dp(d), _dp(nij), _dp(pi), _dp(pj), _dp(g), n)
        return {"i": ci, "j": cj, "dij": d, "nij": nij, "pi": pi, "pj": pj, "gamma": g}

    def lagrange_multiplier(self):
        n = lib().orc_get_lambda(self.h, None, 0)
        out = np.zeros(n)
        lib().orc_get_lambda(self.h, _dp(out), n)
        return out

    def stats(self):
        s = OrcStats()
        lib().orc_get_stats(self.h, C.byref(s))
        return {k: getattr(s, k) for k, _ in OrcStats._fields_}

    def amat(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros(3 * lib().orc_num_contacts(self.h))
        lib().orc_amat(self.h, _dp(u), _dp(out))
        return out

    def atmat(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros(6 * (self.pa.n - self.pa.nb_inactive))
        lib().orc_atmat(self.h, _dp(f), _dp(out))
        return out


def se_record(c, q, r, sq):
    """Body record {c[3], q[4] (w, x, y, z), r[3], e, n} of the superellipsoid entry points."""
    return np.concatenate([np.asarray(c, float).ravel()[:3], np.asarray(q, float).ravel()[:4],
                           np.asarray(r, float).ravel()[:3], np.asarray(sq, float).ravel()[:2]])


def _unpack(out):
    return {"pi": out[0:3].copy(), "pj": out[3:6].copy(), "nij": out[6:9].copy(), "dij": float(out[9]),
            "u": out[10:14].copy(), "nfev": int(out[14])}


def se_se(s1, s2):
    """closest_points(superellipsoid<3>, superellipsoid<3>) on two body records."""
    out = np.zeros(15)
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    info = lib().orc_se_se(_dp(a), _dp(b), _dp(out))
    r = _unpack(out)
    r["info"] = info
    return r


def se_plane(s, plane_c, plane_q):
    """closest_points(superellipsoid<3>, plane<3>); the plane record is {c[3], q[4]}."""
    out = np.zeros(15)
    a = np.ascontiguousarray(s, float)
    p = np.ascontiguousarray(np.concatenate([np.asarray(plane_c, float)[:3], np.asarray(plane_q, float)[:4]]))
    lib().orc_se_plane(_dp(a), _dp(p), _dp(out))
    r = _unpack(out)
    F = np.zeros(4)
    uu = np.ascontiguousarray(r["u"])
    lib().orc_se_plane_residual(_dp(a), _dp(p), _dp(uu), _dp(F))
    r["residual"] = F
    return r


def se_se_system(s1, s2, u):
    """F (4) and the analytic Jacobian (4 x 4) of the SE-SE closest-point system at u."""
    F = np.zeros(4)
    J = np.zeros(16)
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    uu = np.ascontiguousarray(u, float)
    lib().orc_se_se_system(_dp(a), _dp(b), _dp(uu), _dp(F), _dp(J))
    return F, J.reshape(4, 4).T.copy()


def se2_record(c, angle, r, e):
    """2D body record: centre (x, y), rotation angle about z, semi-axes (rx, ry), squareness e."""
    q = [math.cos(angle / 2), 0.0, 0.0, math.sin(angle / 2)]
    return se_record([c[0], c[1], 0.0], q, [r[0], r[1], 0.0], [e, 1.0])


def se2_se2(s1, s2):
    """closest_points(superellipsoid<2>, superellipsoid<2>) on two 2D body records."""
    out = np.zeros(15)
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    info = lib().orc_se2_se2(_dp(a), _dp(b), _dp(out))
    r = _unpack(out)
    r["info"] = info
    r["u"] = r["u"][:2]
    return r


def se2_system(s1, s2, u):
    """F (2) and the analytic Jacobian (2 x 2) of the 2D SE-SE system at u = (b1, b2)."""
    F = np.zeros(2)
    J = np.zeros(4)
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    uu = np.ascontiguousarray(u, float)
    lib().orc_se2_system(_dp(a), _dp(b), _dp(uu), _dp(F), _dp(J))
    return F, J.reshape(2, 2).T.copy()


def hybrid_solve2(s1, s2, u0):
    """The restated MINPACK hybrid method on the 2D SE-SE system from the start u0."""
    u = np.ascontiguousarray(u0, float).copy()
    nfev = C.c_int(0)
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    info = lib().orc_se2_hybrid(_dp(a), _dp(b), _dp(u), C.byref(nfev))
    return {"u": u, "info": info, "nfev": nfev.value}


def se_se_from(s1, s2, u0):
    """closest_points(superellipsoid<3>, superellipsoid<3>) with the solve started from u0."""
    out = np.zeros(15)
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    uu = np.ascontiguousarray(u0, float)
    info = lib().orc_se_se_from(_dp(a), _dp(b), _dp(uu), _dp(out))
    r = _unpack(out)
    r["info"] = info
    return r


def se_se_start_value(s1, s2, u):
    """The start criterion |p1 - p2| + 2 (1 + n1.n2) of the SE-SE solve at angles u."""
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    uu = np.ascontiguousarray(u, float)
    return float(lib().orc_se_se_start_value(_dp(a), _dp(b), _dp(uu)))


def se_se_start(s1, s2):
    """Start (a1, b1, a2, b2) of the SE-SE solve: the first minimum of the start criterion."""
    u = np.zeros(4)
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    lib().orc_se_se_start(_dp(a), _dp(b), _dp(u))
    return u


def hybrid_solve(s1, s2, u0):
    """The restated MINPACK hybrid method on the SE-SE system from the start u0."""
    u = np.ascontiguousarray(u0, float).copy()
    nfev = C.c_int(0)
    a, b = np.ascontiguousarray(s1, float), np.ascontiguousarray(s2, float)
    info = lib().orc_se_se_hybrid(_dp(a), _dp(b), _dp(u), C.byref(nfev))
    return {"u": u, "info": info, "nfev": nfev.value}


def sphere_record(c, q, r):
    """Sphere record {c[3], q[4] (w, x, y, z), radius} of the sphere-superellipsoid entry point."""
    return np.concatenate([np.asarray(c, float).ravel()[:3], np.asarray(q, float).ravel()[:4], [float(r)]])


def sphere_se(dim, se, sph, reference_labels=True, se_is_i=True):
    """closest_points(sphere, superellipsoid) (closest_points.hpp:944-1302 in 3D, 1316-1463 in
    2D) on a superellipsoid record and a sphere record.  reference_labels: the reference's own
    result (pi on the superellipsoid, nij the sphere's unit normal); else the pair labelled by
    body (superellipsoid = body i when se_is_i).  'newton' is the Newton method's return:
    iterations, -1 at the iteration cap, -2 on a singular Jacobian."""
    out = np.zeros(16)
    a, b = np.ascontiguousarray(se, float), np.ascontiguousarray(sph, float)
    info = lib().orc_sphere_se(int(dim), _dp(a), _dp(b), int(bool(reference_labels)), int(bool(se_is_i)), _dp(out))
    r = _unpack(out)
    r["newton"] = info
    if dim == 2:
        r["u"] = r["u"][:2]
    return r


def se2_plane(s, plane_c, plane_angle):
    """closest_points(superellipsoid<2>, plane<2>) in closed form; the plane is (centre, angle)."""
    out = np.zeros(15)
    a = np.ascontiguousarray(s, float)
    q = [np.cos(plane_angle / 2), 0.0, 0.0, np.sin(plane_angle / 2)]
    p = np.ascontiguousarray(np.concatenate([[plane_c[0], plane_c[1], 0.0], q]))
    lib().orc_se2_plane(_dp(a), _dp(p), _dp(out))
    r = _unpack(out)
    r["u"] = r["u"][:2]
    return r


def lu_solve4(A, b):
    """x with A x = b by the Newton method's solve (column-major inside); None on a zero pivot."""
    a = np.ascontiguousarray(np.asarray(A, float).T.ravel())
    bb = np.ascontiguousarray(np.asarray(b, float).ravel())
    x = np.zeros(4)
    rc = lib().orc_lu_solve4(_dp(a), _dp(bb), _dp(x))
    return None if rc else x
