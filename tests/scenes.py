"""Scenes of the reference's own solver tests, rebuilt with scopi_b200.container.

Each builder returns ``(particles, solver_kwargs, dt, total_it)`` with the
settings of the cited reference test (hpc-maths/scopi test/*.cpp).  The default
solver parameters are the reference defaults: dmax 2, kd radius 17
(contact_kdtree.hpp:229-237), apgd alpha 0.05, max_ite 10000, tol 1e-7, dynamic
descent (apgd.hpp:120-123), mu 0.1, gamma 0 / -2 / 1e-6 (property.hpp:72,125-127).
"""
from __future__ import annotations

import math

from scopi_b200.container import Particles, Property, quaternion

PI = math.pi
NOFRICTION, FRICTION, VISCOUS, FRICTION_FIXED_POINT, VISCOUS_FRICTION = 0, 1, 2, 3, 4
VAP_FIXED, VAP_FPD = 0, 1
BRUTE_FORCE, KDTREE = 0, 1


class MinstdRand0:
    """std::minstd_rand0 (a=16807, m=2^31-1) with libstdc++'s uniform_real_distribution<double>.

    libstdc++ generate_canonical<double, 53> draws k=2 values (log2 of the range
    2^31-2 truncates to 30), accumulates (x-1)*r^i in double and divides by the
    double-rounded r^2; the distribution returns canonical*(b-a)+a.
    """

    M = 2147483647

    def __init__(self, seed: int):
        self.x = seed % self.M or 1

    def __call__(self) -> int:
        self.x = (16807 * self.x) % self.M
        return self.x

    def uniform(self, a: float, b: float) -> float:
        r = self.M - 1  # max - min + 1 = (2^31-2) - 1 + 1
        s = float(self() - 1) * 1.0
        s = s + float(self() - 1) * float(r)
        tmp = float(r * r)  # r*r is exact in long double, rounded once to double
        ret = s / tmp
        if ret >= 1.0:
            ret = math.nextafter(1.0, 0.0)
        return ret * (b - a) + a


def contacts_three_disks():
    """test/test_contacts_kdtree.cpp:14-73 (kd radius 100) / test_contacts_brute_force.cpp:12-71."""
    p = Particles(2)
    p.add_sphere((0.0, 0.0), 0.1)
    p.add_sphere((1.0, 1.0), 0.2)
    p.add_sphere((5.0, 10.0), 0.1)
    return p.finalize(), dict(kd_tree_radius=100.0), 0.0, 0


def matrix_a_3d():
    """test/test_matrices.cpp:17-45: two 3D spheres, brute-force contacts, A/A^T adjointness."""
    p = Particles(3)
    p.add_sphere((0.0, 0.0, 0.0), 0.1)
    p.add_sphere((1.0, 1.0, 0.0), 0.2)
    return p.finalize(), dict(contact_method=BRUTE_FORCE), 0.0, 0


def matrix_a_case2():
    """test/test_matrices.cpp:47-77: plane at pi/2-pi/4, sphere (2,1) r=0.5; A.u known values."""
    p = Particles(2)
    p.add_plane((0.0, 0.0), PI / 2 - PI / 4)
    p.add_sphere((2.0, 1.0), 0.5, Property(mass=1, moment_inertia=0.1))
    return p.finalize(), dict(contact_method=BRUTE_FORCE), 0.0, 0


def three_spheres(problem=NOFRICTION):
    """test/test_gradient.cpp:377-642 (NoFriction Tf=6; Viscous, FrictionFixedPoint (mu 0.5,
    fixed point 1e-6 / 1000) and ViscousFriction (mu 0.5, fixed point 1e-3 / 1000, gamma_min -1.4)
    Tf=7; dt 0.1, vap_fpd, alpha 0.1)."""
    p = Particles(2)
    for (x, y) in ((-1.7, 1.3), (0.5, 1.7), (4.5, 1.3)):
        p.add_sphere((x, y), 0.5, Property(mass=1, moment_inertia=1, force=(-x, -y)))
    tf = 6.0 if problem == NOFRICTION else 7.0
    dt = 0.1
    kw = dict(problem=problem, vap=VAP_FPD, contact_method=KDTREE, tolerance=1e-7, max_ite=10000, alpha=0.1)
    if problem == 3:
        kw.update(mu=0.5, fixed_point_tol=1e-6, fixed_point_max_iter=1000)
    if problem == 4:
        kw.update(mu=0.5, fixed_point_tol=1e-3, fixed_point_max_iter=1000, gamma=0.0, gamma_min=-1.4, gamma_tol=1e-6)
    return p.finalize(), kw, dt, int(tf / dt)


def sphere_plane_friction_mu01():
    """test/test_gradient.cpp:156-213: Friction mu 0.1, dt 0.1, Tf 20."""
    p = Particles(2)
    p.add_plane((0.0, 0.0), PI / 2 - PI / 6)
    dd, rr = 1.0, 2.0
    p.add_sphere((0.0, (rr + dd) / math.cos(PI / 6)), rr, Property(mass=1, moment_inertia=0.5 * rr * rr, force=(0, -1)))
    kw = dict(problem=FRICTION, vap=VAP_FPD, contact_method=KDTREE, tolerance=1e-7, max_ite=10000, alpha=0.1, mu=0.1)
    dt = 0.1
    return p.finalize(), kw, dt, int(20 / dt)


def two_spheres(symmetric: bool, contact_method=KDTREE):
    """test/test_sphere.cpp:341-421: vap_fixed, dt 0.005, 1000 steps, default solver."""
    p = Particles(2)
    dy = 0.0 if symmetric else 0.05
    p.add_sphere((-0.2, -dy), 0.1, Property(mass=1.0, moment_inertia=0.1, desired_velocity=(0.25, 0)))
    p.add_sphere((0.2, dy), 0.1, Property(mass=1.0, moment_inertia=0.1, desired_velocity=(-0.25, 0)))
    return p.finalize(), dict(vap=VAP_FIXED, contact_method=contact_method), 0.005, 1000


def critical_2d_spheres(contact_method=KDTREE, n=3, seed=123):
    """test/test_sphere.cpp:423-484: 18 disks from std::minstd_rand0(123), dt 0.01, 20 steps
    (n = 2, seed 0: the 8 disks of test/test_friction.cpp:55-112)."""
    g = MinstdRand0(seed)
    p = Particles(2)
    for i in range(n):
        for j in range(n):
            r = g.uniform(0.2, 0.4)
            x = (i + 0.5) + g.uniform(-0.1, 0.1)
            y = (j + 0.5) + g.uniform(-0.1, 0.1)
            vel = g.uniform(2.0, 5.0)
            p.add_sphere((x, y), r, Property(mass=1.0, moment_inertia=0.1, desired_velocity=(vel, 0.0)))
            r = g.uniform(0.2, 0.4)
            x = (n + i + 0.5) + g.uniform(-0.1, 0.1)
            y = (j + 0.5) + g.uniform(-0.1, 0.1)
            vel = g.uniform(2.0, 5.0)
            p.add_sphere((x, y), r, Property(mass=1.0, moment_inertia=0.1, desired_velocity=(-vel, 0.0)))
    return p.finalize(), dict(vap=VAP_FIXED, contact_method=contact_method), 0.01, 20


def obstacle_sphere_plane(variant: str, contact_method=KDTREE):
    """test/test_obstacles.cpp:43-98: sphere resting on plane(pi/2); variants fixed / velocity / force."""
    p = Particles(2)
    p.add_plane((0.0, 0.0), PI / 2.0)
    prop = Property(mass=1.0, moment_inertia=0.1)
    vap = VAP_FIXED
    if variant == "velocity":
        prop.desired_velocity = (0.0, -1.0)
    elif variant == "force":
        prop.force = (0.0, -1.0)
        vap = VAP_FPD
    p.add_sphere((0.0, 1.0), 1.0, prop)
    return p.finalize(), dict(vap=vap, contact_method=contact_method), 0.005, 100


def obstacle_sphere_sphere(variant: str, contact_method=KDTREE):
    """test/test_obstacles.cpp:100-213: sphere on a fixed sphere; fixed / velocity / force / moving."""
    p = Particles(2)
    p.add_sphere((0.0, 0.0), 1.0, Property().deactivate())
    prop = Property(mass=1.0, moment_inertia=0.1)
    vap = VAP_FIXED
    pos = (0.0, 2.0)
    if variant == "velocity":
        prop.desired_velocity = (0.0, -1.0)
    elif variant == "force":
        prop.force = (0.0, -1.0)
        vap = VAP_FPD
    elif variant == "moving":
        pos = (1.0, math.sqrt(3.0))
        prop.force = (0.0, -10.0)
        vap = VAP_FPD
    p.add_sphere(pos, 1.0, prop)
    return p.finalize(), dict(vap=vap, contact_method=contact_method), 0.005, 100


def sphere_inclined_plane(alpha: float, contact_method=KDTREE):
    """test/test_obstacles.cpp:252-311: plane at pi/2-alpha, g=1, dt 0.01, 1000 steps, vap_fpd."""
    radius, g, h = 1.0, 1.0, 2.0
    p = Particles(2)
    p.add_plane((0.0, 0.0), PI / 2.0 - alpha)
    p.add_sphere((h * math.sin(alpha), h * math.cos(alpha)), radius,
                 Property(mass=1.0, moment_inertia=1.0 * radius * radius / 2.0, force=(0.0, -g)))
    return p.finalize(), dict(vap=VAP_FPD, contact_method=contact_method), 0.01, 1000


def sphere_plane_analytic(problem=NOFRICTION):
    """test/test_gradient.cpp:23-154: sphere on plane(pi/2), tilted gravity g(sin a, -cos a), a=pi/4."""
    radius, g, h, alpha = 1.0, 1.0, 2.0, PI / 4
    p = Particles(2)
    p.add_plane((0.0, 0.0), PI / 2)
    p.add_sphere((0.0, h), radius, Property(mass=1, moment_inertia=radius * radius / 2.0,
                                            force=(g * math.sin(alpha), -g * math.cos(alpha))))
    if problem == NOFRICTION:
        kw = dict(problem=NOFRICTION, vap=VAP_FPD, tolerance=1e-7, max_ite=10000, alpha=0.01)
        return p.finalize(), kw, 0.01, 1000
    kw = dict(problem=VISCOUS, vap=VAP_FPD, tolerance=1e-7, max_ite=10000, alpha=0.1)
    return p.finalize(), kw, 0.01, 500


def analytic_no_friction(alpha, t, r, g, y0):
    """test/analytical_solution.cpp:6-37."""
    t_imp = math.sqrt(2 * (y0 - r) / (g * math.cos(alpha)))
    if t < t_imp:
        x = (g * t ** 2 * math.sin(alpha) / 2, -g * t ** 2 * math.cos(alpha) / 2 + y0)
        v = (g * t * math.sin(alpha), -g * t * math.cos(alpha))
    else:
        x = (g * t ** 2 * math.sin(alpha) / 2, r)
        v = (g * t * math.sin(alpha), 0.0)
    return x, v


def analytic_viscous(alpha, t, r, g, y0, gamma_min, t_inv):
    """test/analytical_solution.cpp:39-124 (position and velocity)."""
    t_imp = math.sqrt(2 * (y0 - r) / (g * math.cos(alpha)))
    t_gmin = -gamma_min / (g * math.cos(alpha))
    gamma_inv = gamma_min if t_inv > t_gmin else -g * t_inv * math.cos(alpha)
    t_unstick = t_inv - gamma_inv / (g * math.cos(alpha))
    sa, ca = math.sin(alpha), math.cos(alpha)
    if t < t_imp:
        return (g * t ** 2 * sa / 2, -g * t ** 2 * ca / 2 + y0), (g * t * sa, -g * t * ca)
    if t < t_inv:
        return (g * t ** 2 * sa / 2, r), (g * t * sa, 0.0)
    xs = g * t_inv ** 2 * sa / 2 + g * t_inv * sa * (t - t_inv) - g * (t - t_inv) ** 2 * sa / 2
    vx = g * t_inv * sa - g * (t - t_inv) * sa
    if t < t_unstick:
        return (xs, r), (vx, 0.0)
    return (xs, r + g * (t - t_unstick) ** 2 * ca / 2), (vx, g * (t - t_unstick) * ca)


def analytic_inclined(alpha, mu, t, r, g, y0):
    """test/utils.cpp:77-139 (position, theta) and velocity."""
    t_imp = math.sqrt(2 * (y0 - r) / (g * math.cos(alpha)))
    sa, ca = math.sin(alpha), math.cos(alpha)
    if t > t_imp:
        vtm = g * t_imp * sa
        vnm = -g * t_imp * ca
        t2 = t - t_imp
        x_imp = g * sa * t_imp * t_imp / 2.0
        if math.tan(alpha) <= 3 * mu:
            xn = g * sa * t2 * t2 / 3.0 + 2.0 * vtm * t2 / 3.0 + x_imp
            theta = -g * sa * t2 * t2 / (3.0 * r) - 2 * vtm * t2 / (3.0 * r)
            vn = 2.0 * g * sa * t2 / 3.0 + 2.0 * vtm / 3.0
        else:
            xn = g * (sa - mu * ca) * t2 * t2 / 2.0 + (vtm + mu * vnm) * t2 + x_imp
            theta = -mu * g * ca * t2 * t2 / r + 2 * mu * vnm * t2 / r
            vn = g * (sa - mu * ca) * t2 + (vtm + mu * vnm)
        x = (xn * ca + r * sa, -xn * sa + r * ca)
        v = (vn * ca, -vn * sa)
        return x, theta, v
    return (y0 * sa, y0 * ca - g * t * t / 2.0), 0.0, (0.0, -g * t)


__all__ = ["quaternion"]


def two_ellipsoids(semi_y: float, dy: float, total_it: int):
    """test/test_superellipsoid.cpp:451-628: two 2D superellipsoids (e = 1) at (-0.2, -dy) and
    (0.2, dy), rotated by +-pi/4, semi-axes (0.1, semi_y), desired velocities +-0.25, vap_fixed,
    dt 0.005, default solver.  symmetrical: dy 0, 200 steps (semi_y 0.05) or 50 (semi_y 0.1);
    asymmetrical: dy 0.05, 1000 steps."""
    p = Particles(2)
    p.add_superellipsoid((-0.2, -dy), (0.1, semi_y), 1.0,
                         Property(mass=1.0, moment_inertia=0.1, desired_velocity=(0.25, 0)), q=quaternion(PI / 4))
    p.add_superellipsoid((0.2, dy), (0.1, semi_y), 1.0,
                         Property(mass=1.0, moment_inertia=0.1, desired_velocity=(-0.25, 0)), q=quaternion(-PI / 4))
    return p.finalize(), dict(vap=VAP_FIXED, contact_method=KDTREE), 0.005, total_it


def critical_2d_superellipsoids():
    """test/test_superellipsoid.cpp:630-702: 18 2D superellipsoids (e = 1) from
    std::minstd_rand0(123), dt 0.01, 20 steps, default solver."""
    n = 3
    g = MinstdRand0(123)
    p = Particles(2)
    for i in range(n):
        for j in range(n):
            for side in (0, 1):
                rot = g.uniform(0.0, PI)
                r = g.uniform(0.2, 0.4)
                r2 = g.uniform(0.2, 0.4)
                x = (side * n + i + 0.5) + g.uniform(-0.1, 0.1)
                y = (j + 0.5) + g.uniform(-0.1, 0.1)
                vel = g.uniform(2.0, 5.0)
                p.add_superellipsoid((x, y), (r, r2), 1.0,
                                     Property(mass=1.0, moment_inertia=0.1,
                                              desired_velocity=(vel if side == 0 else -vel, 0.0)),
                                     q=quaternion(rot))
    return p.finalize(), dict(vap=VAP_FIXED, contact_method=KDTREE), 0.01, 20


def sphere_plane_fixed_point():
    """test/test_gradient.cpp:215-283: FrictionFixedPoint, sphere on plane(pi/2) under tilted gravity
    g(sin a, -cos a), a = pi/4, mu 0.5, fixed point tol 1e-6 / 1000, dt 0.01, 500 steps, vap_fpd."""
    radius, g, h, alpha = 1.0, 1.0, 2.0, PI / 4
    p = Particles(2)
    p.add_plane((0.0, 0.0), PI / 2)
    p.add_sphere((0.0, h), radius, Property(mass=1, moment_inertia=radius * radius / 2.0,
                                            force=(g * math.sin(alpha), -g * math.cos(alpha))))
    kw = dict(problem=3, vap=VAP_FPD, tolerance=1e-7, max_ite=10000, alpha=0.01, mu=0.5, fixed_point_tol=1e-6,
              fixed_point_max_iter=1000)
    return p.finalize(), kw, 0.01, 500


def analytic_friction(alpha, mu, t, r, g, y0):
    """test/analytical_solution.cpp:130-187: position, angle, velocity and angular velocity of the
    sphere on the plane under tilted gravity, with friction mu."""
    t_imp = math.sqrt(2 * (y0 - r) / (g * math.cos(alpha)))
    sa, ca = math.sin(alpha), math.cos(alpha)
    if t <= t_imp:
        return (g * t * t * sa / 2, -g * t * t * ca / 2 + y0), 0.0, (g * t * sa, -g * t * ca), 0.0
    vtm, vnm = g * t_imp * sa, -g * t_imp * ca
    t2 = t - t_imp
    x_imp = g * t_imp * t_imp * sa / 2
    if math.tan(alpha) <= 3 * mu:
        x = g * sa * t2 * t2 / 3.0 + 2.0 * vtm * t2 / 3.0 + x_imp
        theta = -g * sa * t2 * t2 / (3.0 * r) - 2 * vtm * t2 / (3.0 * r)
        v = 2.0 * g * sa * t2 / 3.0 + 2.0 * vtm / 3.0
        om = -2.0 * g * sa * t2 / (3.0 * r) - 2 * vtm / (3.0 * r)
    else:
        x = g * (sa - mu * ca) * t2 * t2 / 2.0 + (vtm + mu * vnm) * t2 + x_imp
        theta = -mu * g * ca * t2 * t2 / r + 2 * mu * vnm * t2 / r
        v = g * (sa - mu * ca) * t2 + (vtm + mu * vnm)
        om = -2.0 * mu * g * ca * t2 / r + 2 * mu * vnm / r
    return (x, r), theta, (v, 0.0), om


def sphere_plane_viscous_friction():
    """test/test_gradient.cpp:284-372: ViscousFriction, sphere on plane(pi/2) under tilted gravity
    g(sin a, -cos a), a = pi/4, mu 0.5, fixed point 1e-3 / 1000, gamma 0, gamma_min -1.4, gamma_tol
    1e-6, alpha 0.1, dt 0.01: 500 steps, then the force flipped for 100 more."""
    radius, g, h, alpha = 1.0, 1.0, 2.0, PI / 4
    p = Particles(2)
    p.add_plane((0.0, 0.0), PI / 2)
    p.add_sphere((0.0, h), radius, Property(mass=1, moment_inertia=radius * radius / 2.0,
                                            force=(g * math.sin(alpha), -g * math.cos(alpha))))
    kw = dict(problem=VISCOUS_FRICTION, vap=VAP_FPD, tolerance=1e-7, max_ite=10000, alpha=0.1, mu=0.5,
              fixed_point_tol=1e-3, fixed_point_max_iter=1000, gamma=0.0, gamma_min=-1.4, gamma_tol=1e-6)
    return p.finalize(), kw, 0.01, 500


def analytic_viscous_friction(alpha, mu, t, r, g, y0, gamma_min, t_inv):
    """test/analytical_solution.cpp:193-417: the sphere falls, sticks, slides with friction once the
    adhesion potential has reached gamma_min (rolling without slip after t_no_slide when
    tan a <= 3 mu), and after the force flips at t_inv moves back and unsticks.
    Returns position, angle, velocity, angular velocity.  The reference's velocity branch writes
    t_no_slide as -tan(a) t_gm / (g (tan a - 3 mu)) + t_gm and its position branch as
    -v_gm / (g cos(a) (tan a - 3 mu)) + t_gm (equal when g = 1); both are kept."""
    sa, ca, ta = math.sin(alpha), math.cos(alpha), math.tan(alpha)
    t_imp = math.sqrt(2 * (y0 - r) / (g * ca))
    t_gm = -gamma_min / (g * ca)
    gamma_inv = gamma_min if t_inv > t_gm else -g * t_inv * ca
    if t < t_imp:
        return (g * t * t * sa / 2, -g * t * t * ca / 2 + y0), 0.0, (g * t * sa, -g * t * ca), 0.0
    if t < t_gm:
        return (g * t * t * sa / 2, r), 0.0, (g * t * sa, 0.0), 0.0
    v_gm = -gamma_min * ta
    x_gm = g * t_gm * t_gm * sa / 2

    def slide(tt):
        """(x, angle, v, omega) while sliding at gamma_min, tt >= t_gm."""
        t2 = tt - t_gm
        return (g * (sa - mu * ca) * t2 * t2 / 2 + v_gm * t2 + x_gm, -mu * g * ca * t2 * t2 / r,
                g * (sa - mu * ca) * t2 + v_gm, -2.0 * mu * g * ca * t2 / r)

    def state(tt):
        """(x, angle, v, omega) at gamma_min before the flip, rolling after t_no_slide."""
        out = list(slide(tt))
        if ta > 3 * mu:
            return out
        t_ns_x = -v_gm / (g * ca * (ta - 3 * mu)) + t_gm
        t_ns_v = -ta * t_gm / (g * (ta - 3 * mu)) + t_gm
        if tt > t_ns_x:
            x_ns, a_ns, v_ns, w_ns = slide(t_ns_x)
            t3 = tt - t_ns_x
            out[0] = g * sa * t3 * t3 / 3.0 + v_ns * t3 + x_ns
            out[1] = -g * sa * t3 * t3 / (3.0 * r) + w_ns * t3 + a_ns
        if tt > t_ns_v:
            _, _, v_ns, w_ns = slide(t_ns_v)
            t3 = tt - t_ns_v
            out[2] = 2.0 * g * sa * t3 / 3.0 + v_ns
            out[3] = -2.0 * g * sa * t3 / (3.0 * r) + w_ns
        return out

    if t < t_inv:
        x, ang, vx, w = state(t)
        return (x, r), ang, (vx, 0.0), w
    x_i, a_i, v_i, w_i = state(t_inv)
    t_unstick = t_inv - gamma_inv / (g * ca)
    t4 = t - t_inv
    x = v_i * t4 - g * sa * t4 * t4 / 2 + x_i
    ang = w_i * t4 + a_i
    vx = v_i - g * sa * t4
    if t < t_unstick:
        y, vy = r, 0.0
    else:
        y, vy = g * ca * (t - t_unstick) ** 2 / 2 + r, g * ca * (t - t_unstick)
    return (x, y), ang, (vx, vy), w_i


def viscous_friction_3d(mu=0.3, gamma_min=-0.03):
    """ViscousFriction in 3D: a 3x3 layer of touching spheres (r 0.5) on the floor plane z = 0
    with a 2x2 layer in its pockets, under gravity tilted by pi/6 along x, vap_fpd, dt 0.01.
    The floor contacts pass through the viscous pair to gamma_min within a few steps, then
    slide on the friction cone."""
    p = Particles(3)
    p.add_plane((0.0, 0.0, 0.0), q=quaternion(PI / 2, (0, 1, 0)))
    r, a = 0.5, PI / 6
    prop = dict(mass=1.0, moment_inertia=(0.1, 0.1, 0.1), force=(math.sin(a), 0.0, -math.cos(a)))
    for i in range(3):
        for j in range(3):
            p.add_sphere((float(i), float(j), r), r, Property(**prop))
    z2 = r + math.sqrt(0.5)
    for i in range(2):
        for j in range(2):
            p.add_sphere((i + 0.5, j + 0.5, z2), r, Property(**prop))
    kw = dict(problem=VISCOUS_FRICTION, vap=VAP_FPD, tolerance=1e-7, max_ite=10000, alpha=0.1, mu=mu, dmax=0.1,
              fixed_point_tol=1e-3, fixed_point_max_iter=1000, gamma=0.0, gamma_min=gamma_min, gamma_tol=1e-6)
    return p.finalize(), kw, 0.01, 40


def two_worms(contact_method=KDTREE):
    """test/test_worm.cpp:480-530: two 2D worms of six unit spheres (mass 1, moment of inertia
    0.1) driven into each other by vap_fixed at desired velocities (-1, 0) and (1, 0),
    NoFriction, dmax 1, default solver parameters, dt 0.005, 1000 steps."""
    p = Particles(2)
    prop = dict(mass=1.0, moment_inertia=0.1)
    p.add_worm([(1.0 + 2 * k, 0.7) for k in range(6)], 1.0, Property(desired_velocity=(-1.0, 0.0), **prop))
    p.add_worm([(-1.0 - 2 * k, -0.7) for k in range(6)], 1.0, Property(desired_velocity=(1.0, 0.0), **prop))
    kw = dict(problem=NOFRICTION, vap=VAP_FIXED, contact_method=contact_method, dmax=1.0)
    return p.finalize(), kw, 0.005, 1000


def periodic_disks(problem=NOFRICTION, contact_method=KDTREE):
    """A periodic BoxDomain (box.hpp) along x, [0, 4]: two rows of eight disks (r 0.2) on a
    horizontal floor plane whose position (x = 2) stays away from the periodic bound, the
    lower row moving at +1, the upper at -0.6, gravity -1, vap_fpd, dmax 0.3, dt 0.01, 150
    steps; the rows cross the bound several times and meet their copies."""
    p = Particles(2)
    p.add_plane((2.0, 0.0), PI / 2)
    for k in range(8):
        p.add_sphere((0.25 + 0.5 * k, 0.2), 0.2, Property(mass=1.0, moment_inertia=0.02, velocity=(1.0, 0.0),
                                                          force=(0.0, -1.0)))
    for k in range(8):
        p.add_sphere((0.5 * k, 0.6), 0.2, Property(mass=1.0, moment_inertia=0.02, velocity=(-0.6, 0.0),
                                                   force=(0.0, -1.0)))
    kw = dict(problem=problem, vap=VAP_FPD, contact_method=contact_method, dmax=0.3, tolerance=1e-9,
              max_ite=20000, alpha=0.1, box_lower=(0.0, 0.0, 0.0), box_upper=(4.0, 0.0, 0.0), periodic=(1, 0, 0))
    if problem == FRICTION:
        kw["mu"] = 0.3
    return p.finalize(), kw, 0.01, 150


def periodic_two_disks(unwrapped=False):
    """Two disks (r 0.25) meeting across the periodic bound x = 0 of the box [0, 4]: A at 0.3
    moving at -0.5, B at 3.7 moving at +0.5 (vap_fixed, dmax 0.5, so that A's copy joins the
    search); with ``unwrapped`` the same scene without a box, B at 3.7 - 4."""
    p = Particles(2)
    p.add_sphere((0.3, 0.0), 0.25, Property(mass=1.0, moment_inertia=0.1, desired_velocity=(-0.5, 0.0)))
    p.add_sphere((-0.3 if unwrapped else 3.7, 0.0), 0.25, Property(mass=1.0, moment_inertia=0.1,
                                                                   desired_velocity=(0.5, 0.0)))
    kw = dict(problem=NOFRICTION, vap=VAP_FIXED, dmax=0.5, tolerance=1e-10, max_ite=20000, alpha=0.1)
    if not unwrapped:
        kw.update(box_lower=(0.0, 0.0, 0.0), box_upper=(4.0, 0.0, 0.0), periodic=(1, 0, 0))
    return p.finalize(), kw, 0.01, 40


def periodic_spheres_3d(problem=NOFRICTION):
    """A 3D box periodic along x, [0, 2]: a 4 x 4 layer of spheres (r 0.2) on the floor plane
    z = 0 (its position x = 1 away from the bound) sliding at (1, 0.3, 0) under gravity -z,
    vap_fpd, dmax 0.3, dt 0.01, 100 steps."""
    p = Particles(3)
    p.add_plane((1.0, 0.5, 0.0), q=quaternion(PI / 2, (0, 1, 0)))
    for i in range(4):
        for j in range(4):
            p.add_sphere((0.25 + 0.5 * i, 0.25 + 0.45 * j, 0.2), 0.2,
                         Property(mass=1.0, moment_inertia=(0.016, 0.016, 0.016), velocity=(1.0, 0.3, 0.0),
                                  force=(0.0, 0.0, -1.0)))
    kw = dict(problem=problem, vap=VAP_FPD, dmax=0.3, tolerance=1e-9, max_ite=20000, alpha=0.1,
              box_lower=(0.0, 0.0, 0.0), box_upper=(2.0, 0.0, 0.0), periodic=(1, 0, 0))
    if problem == FRICTION:
        kw["mu"] = 0.3
    return p.finalize(), kw, 0.01, 100


def two_spheres_friction(contact_method=KDTREE):
    """test/test_friction.cpp:17-53: two disks (r 0.1) pushed into each other off-centre by
    vap_fixed at (0.25, 0) and (-0.25, 0), Friction mu 0.5, default solver, dt 0.005; the
    reference's snapshot is the state after 999 steps."""
    p = Particles(2)
    p.add_sphere((-0.2, -0.05), 0.1, Property(mass=1.0, moment_inertia=0.1, desired_velocity=(0.25, 0.0)))
    p.add_sphere((0.2, 0.05), 0.1, Property(mass=1.0, moment_inertia=0.1, desired_velocity=(-0.25, 0.0)))
    return p.finalize(), dict(problem=FRICTION, vap=VAP_FIXED, contact_method=contact_method, mu=0.5), 0.005, 999


def critical_2d_spheres_friction(contact_method=KDTREE):
    """test/test_friction.cpp:55-112: the critical 2D disks (n = 2, std::minstd_rand0(0)),
    Friction mu 0.5, vap_fixed, dt 0.01; the reference's snapshot is the state after 99 steps."""
    pa, _, dt, _ = critical_2d_spheres(contact_method, n=2, seed=0)
    return pa, dict(problem=FRICTION, vap=VAP_FIXED, contact_method=contact_method, mu=0.5), dt, 99
