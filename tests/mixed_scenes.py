"""Scenes of spheres and superellipsoids together (the sphere-superellipsoid pairs of
closest_points.hpp:944-1463 and the 2D superellipsoid-plane pairs of :1783-1958): seeded
jittered lattices, half spheres and half superellipsoids, above a plane floor (3D) or in a
box of four planes (2D), under gravity."""
from __future__ import annotations

import math

import numpy as np

from scopi_b200.container import Particles, Property, quaternion


def random_q(rng):
    """Uniform random rotation (Shoemake), as (w, x, y, z)."""
    u = rng.uniform(size=3)
    return np.array([math.sqrt(u[0]) * math.cos(2 * math.pi * u[2]), math.sqrt(1 - u[0]) * math.sin(2 * math.pi * u[1]),
                     math.sqrt(1 - u[0]) * math.cos(2 * math.pi * u[1]), math.sqrt(u[0]) * math.sin(2 * math.pi * u[2])])


def mixed_pile_3d(side=5, seed=3, scale=1.0):
    """side^3 bodies on a jittered lattice (spacing 18 mm) above the plane z = 0 (normal +z):
    spheres of radius U[4, 8] mm and superellipsoids of semi-axes U[4, 8] mm, squareness
    U[0.6, 1.4], random orientation, chosen by a fair coin; mass 1, inertia 1e-5, force
    (0, 0, -1).  scale multiplies every length (scale 25: bodies of 0.1-0.2, the size of the
    reference's own closest-point tests)."""
    rng = np.random.default_rng(seed)
    p = Particles(3)
    p.add_plane((0.0, 0.0, 0.0), q=quaternion(-math.pi / 2, (0, 1, 0)))
    prop = dict(mass=1.0, moment_inertia=(1e-5, 1e-5, 1e-5), force=(0.0, 0.0, -1.0))
    spacing = 0.018 * scale
    for k in range(side ** 3):
        x, y, z = k % side, (k // side) % side, k // (side * side)
        c = np.array([(x - side / 2) * spacing, (y - side / 2) * spacing, (0.011 + z * 0.018) * scale])
        c += rng.uniform(-0.002, 0.002, 3) * scale
        if rng.uniform() < 0.5:
            p.add_sphere(c, rng.uniform(0.004, 0.008) * scale, Property(**prop))
        else:
            p.add_superellipsoid(c, rng.uniform(0.004, 0.008, 3) * scale, rng.uniform(0.6, 1.4, 2), Property(**prop),
                                 q=random_q(rng))
    return p.finalize()


def mixed_box_2d(side=8, seed=5, spacing=0.018):
    """side^2 disks and 2D superellipsoids (semi-axes U[4, 8] mm, squareness U[0.6, 1.4], random
    angle) on a jittered lattice inside four planes (the box [-L, L] x [0, 2L]); gravity -y."""
    rng = np.random.default_rng(seed)
    p = Particles(2)
    half = side * spacing / 2 + 0.01
    p.add_plane((0.0, 0.0), math.pi / 2)        # floor y = 0, normal +y
    p.add_plane((-half, 0.0), 0.0)              # left wall, normal +x
    p.add_plane((half, 0.0), math.pi)           # right wall, normal -x
    p.add_plane((0.0, 2 * half), -math.pi / 2)  # ceiling, normal -y
    prop = dict(mass=1.0, moment_inertia=1e-5, force=(0.0, -1.0, 0.0))
    for k in range(side * side):
        x, y = k % side, k // side
        c = np.array([(x - side / 2 + 0.5) * spacing, 0.011 + y * spacing]) + rng.uniform(-0.002, 0.002, 2)
        if rng.uniform() < 0.5:
            p.add_sphere(c, rng.uniform(0.004, 0.008), Property(**prop))
        else:
            a = rng.uniform(0, 2 * math.pi)
            p.add_superellipsoid(c, rng.uniform(0.004, 0.008, 2), [rng.uniform(0.6, 1.4)], Property(**prop),
                                 q=quaternion(a))
    return p.finalize()
