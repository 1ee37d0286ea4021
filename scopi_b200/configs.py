"""Seeded synthetic workloads (SplitMix64 -> uniform doubles), shared by tests and bench.

Generator: SplitMix64 with state_k = seed + (k+1) * 0x9E3779B97F4A7C15 (mod 2^64), the
usual three xor-shift-multiply rounds, uniform = (z >> 11) * 2^-53.  Draw order is
stated per workload so any implementation can rebuild the same inputs.

Workloads (shapes and distributions of the benchmark configurations):
  disks_2d        1024 disks, radius U[0.008,0.012], 32x32 grid spacing 0.025, jitter +-0.002,
                  desired velocity -0.25 (x-c)/|x-c| toward c=(0.4,0.4), m=1, J=0.1.
  box_3d          spheres on a jittered 47^3 lattice (spacing 0.0115, jitter +-0.0005),
                  radius U[0.9,1.1]*0.005, m=(r/0.005)^3, J=0.4 m r^2, gravity -9.81 m in z,
                  six fixed planes bounding the unit box.
  pile_scenes     independent 2D scenes for the batched solve: N_s = round(exp(U[ln 200, ln 5000]))
                  disks, radius U[0.008,0.012], random sequential non-overlapping placement in
                  [0,W] x [0.02, 0.02+H], W = H = 0.04 sqrt(N_s), a fixed segment (0,0)-(W,0)
                  below, m = (r/0.01)^2, J = m r^2 / 2, gravity -9.81 m.
  spheres_1m      100^3 spheres on a jittered lattice (spacing 0.0045, jitter +-0.0002) centred
                  in the unit box, radius U[0.9,1.1]*0.002, desired velocity 0.1 (c-x)/|c-x|,
                  m=(r/0.002)^3, J=0.4 m r^2, six plane walls.
  se_pile         3D superellipsoids on the first `count` points of a side^3 lattice (spacing
                  0.018, centred in x and y, lowest layer at z = 0.02; k fastest), semi-axes
                  U[0.004,0.008] each, squareness e, n U[0.6,1.4], uniform random orientation
                  (Shoemake), m = abc/0.006^3, J = m/5 (b^2+c^2, a^2+c^2, a^2+b^2), gravity
                  -9.81 m in z, a floor plane z = 0 with its normal +z.
"""
from __future__ import annotations

import math

import numpy as np

from .container import PLANE, SPHERE, ParticleArrays, quaternion

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix_uniform(seed: int, n: int) -> np.ndarray:
    """n uniforms in [0,1) from SplitMix64(seed)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * _G
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def _arrays(dim, shape, pos, q, v, omega, vd, omega_d, f, m, j, radius, length, nin):
    return ParticleArrays(dim=dim, nb_inactive=nin, shape=np.ascontiguousarray(shape, np.int32),
                          pos=np.ascontiguousarray(pos), q=np.ascontiguousarray(q), v=np.ascontiguousarray(v),
                          omega=np.ascontiguousarray(omega), vd=np.ascontiguousarray(vd),
                          omega_d=np.ascontiguousarray(omega_d), f=np.ascontiguousarray(f), m=np.ascontiguousarray(m),
                          j=np.ascontiguousarray(j), radius=np.ascontiguousarray(radius),
                          length=np.ascontiguousarray(length))


def _box_planes():
    """Six planes of the unit box; normal = column 0 of R(q) (plane.hpp:143-147)."""
    zq = quaternion(0.0, (0, 0, 1))
    yq = quaternion(math.pi / 2, (0, 0, 1))
    xq = quaternion(math.pi / 2, (0, 1, 0))
    pos = [(0, 0, 0), (1, 0, 0), (0, 0, 0), (0, 1, 0), (0, 0, 0), (0, 0, 1)]
    qs = [zq, zq, yq, yq, xq, xq]
    return np.array(pos, dtype=np.float64), np.array(qs)


def _assemble(dim, centers, radius, m, jm, vd=None, f=None, planes=True):
    n_a = len(radius)
    if planes:
        ppos, pq = _box_planes()
        nin = len(ppos)
    else:
        ppos, pq, nin = np.zeros((0, 3)), np.zeros((0, 4)), 0
    n = nin + n_a
    shape = np.full(n, SPHERE, np.int32)
    shape[:nin] = PLANE
    pos = np.zeros((n, 3))
    pos[:nin] = ppos
    pos[nin:, :dim] = centers[:, :dim]
    q = np.zeros((n, 4))
    q[:, 0] = 1.0
    q[:nin] = pq
    z3 = np.zeros((n, 3))
    vdd = z3.copy()
    if vd is not None:
        vdd[nin:, :dim] = vd[:, :dim]
    ff = z3.copy()
    if f is not None:
        ff[nin:, :dim] = f[:, :dim]
    mm = np.ones(n)
    mm[nin:] = m
    jj = np.ones((n, 3))
    jj[nin:] = jm
    rr = np.zeros(n)
    rr[nin:] = radius
    return _arrays(dim, shape, pos, q, z3.copy(), z3.copy(), vdd, z3.copy(), ff, mm, jj, rr, np.zeros(n), nin)


def disks_2d(seed: int = 1, side: int = 32) -> ParticleArrays:
    """Draws per disk k = i*side + j: jitter x, jitter y, radius."""
    n = side * side
    u = splitmix_uniform(seed, 3 * n).reshape(n, 3)
    ii, jj = np.meshgrid(np.arange(side), np.arange(side), indexing="ij")
    cx = 0.0125 + 0.025 * ii.ravel() + (u[:, 0] * 2 - 1) * 0.002
    cy = 0.0125 + 0.025 * jj.ravel() + (u[:, 1] * 2 - 1) * 0.002
    r = 0.008 + (0.012 - 0.008) * u[:, 2]
    c = np.array([0.4, 0.4])
    x = np.stack([cx, cy], 1)
    d = x - c
    nrm = np.sqrt((d * d).sum(1))
    nrm[nrm == 0] = 1.0
    vd = -0.25 * d / nrm[:, None]
    jm = np.zeros((n, 3))
    jm[:, 2] = 0.1
    return _assemble(2, x, r, np.ones(n), jm, vd=vd, planes=False)


def _lattice(seed, count, side, spacing, origin, jitter, r0):
    """Draws per sphere k (lexicographic, k fastest): jitter x, y, z, radius."""
    u = splitmix_uniform(seed, 4 * count).reshape(count, 4)
    idx = np.arange(count)
    ix, iy, iz = idx // (side * side), (idx // side) % side, idx % side
    c = np.stack([origin[0] + spacing * ix, origin[1] + spacing * iy, origin[2] + spacing * iz], 1)
    c = c + (u[:, :3] * 2 - 1) * jitter
    r = (0.9 + 0.2 * u[:, 3]) * r0
    return c, r


def box_3d(seed: int = 2, count: int = 100_000, side: int = 47) -> ParticleArrays:
    sp = 0.0115
    origin = (0.5 - 23 * sp, 0.5 - 23 * sp, sp)
    c, r = _lattice(seed, count, side, sp, origin, 0.0005, 0.005)
    m = (r / 0.005) ** 3
    jm = np.repeat((0.4 * m * r * r)[:, None], 3, 1)
    f = np.zeros((count, 3))
    f[:, 2] = -9.81 * m
    return _assemble(3, c, r, m, jm, f=f)


def spheres_1m(seed: int = 5, side: int = 100) -> ParticleArrays:
    sp = 0.0045
    count = side ** 3
    o = 0.5 - (side - 1) / 2 * sp
    c, r = _lattice(seed, count, side, sp, (o, o, o), 0.0002, 0.002)
    m = (r / 0.002) ** 3
    jm = np.repeat((0.4 * m * r * r)[:, None], 3, 1)
    d = np.array([0.5, 0.5, 0.5]) - c
    nrm = np.sqrt((d * d).sum(1))
    nrm[nrm == 0] = 1.0
    vd = 0.1 * d / nrm[:, None]
    return _assemble(3, c, r, m, jm, vd=vd)


def se_pile(count: int = 50_000, side: int = 37, seed: int = 3) -> ParticleArrays:
    """Draws per body k: semi-axes (3), squareness e, n (2), Shoemake u1, u2, u3 (3)."""
    from .container import Particles, Property
    u = splitmix_uniform(seed, 8 * count).reshape(count, 8)
    sp = 0.018
    p = Particles(3)
    p.add_plane((0.0, 0.0, 0.0), q=quaternion(-math.pi / 2, (0, 1, 0)))  # normal (column 0 of R) = +z
    for k in range(count):
        ix, iy, iz = k // (side * side), (k // side) % side, k % side
        c = ((ix - (side - 1) / 2) * sp, (iy - (side - 1) / 2) * sp, 0.02 + iz * sp)
        a, b, cc = 0.004 + 0.004 * u[k, 0:3]
        e, n = 0.6 + 0.8 * u[k, 3:5]
        u1, u2, u3 = u[k, 5:8]
        q = np.array([math.sqrt(u1) * math.cos(2 * math.pi * u3), math.sqrt(1 - u1) * math.sin(2 * math.pi * u2),
                      math.sqrt(1 - u1) * math.cos(2 * math.pi * u2), math.sqrt(u1) * math.sin(2 * math.pi * u3)])
        m = a * b * cc / 0.006 ** 3
        prop = Property(mass=m, moment_inertia=(m / 5 * (b * b + cc * cc), m / 5 * (a * a + cc * cc),
                                                m / 5 * (a * a + b * b)), force=(0.0, 0.0, -9.81 * m))
        p.add_superellipsoid(c, (a, b, cc), (e, n), prop, q=q)
    return p.finalize()


def se_kd_radius(pa: ParticleArrays, dmax: float) -> float:
    """Squared kd-tree candidate radius (2 r_max + dmax)^2 with r_max the largest bounding
    radius of the active bodies (the search radius of the reference's contact_kdtree)."""
    return float((2 * pa.radius[pa.nb_inactive:].max() + dmax) ** 2)


def pile_scene(seed: int, nmin: int = 200, nmax: int = 5000, vmax: float = 0.0) -> ParticleArrays:
    """One pile scene.  Draws: u[0] -> N_s; candidate k uses (x, y, r) = u[1+3k], u[2+3k], u[3+3k].

    vmax > 0 gives the disks initial velocities U[-vmax, vmax]^2 (draws 2k, 2k+1 of
    SplitMix64(seed + 0x5851F42D), disk k in placement order), so that neighbours approach
    each other and the first steps already have active constraints (tests, profiles)."""
    from .container import Particles, Property
    n_draw = 1 + 3 * 16 * nmax
    u = splitmix_uniform(seed, n_draw)
    n = int(round(math.exp(math.log(nmin) + u[0] * (math.log(nmax) - math.log(nmin)))))
    W = H = 0.04 * math.sqrt(n)
    cell = 0.025
    grid = {}
    placed = []
    k = 0
    while len(placed) < n:
        if 3 + 3 * k >= len(u):
            u = splitmix_uniform(seed, 2 * len(u))
            if k > 400 * n:
                break
        x = u[1 + 3 * k] * W
        y = 0.02 + u[2 + 3 * k] * H
        r = 0.008 + 0.004 * u[3 + 3 * k]
        k += 1
        ci, cj = int(x // cell), int(y // cell)
        ok = True
        for a in (ci - 1, ci, ci + 1):
            for b in (cj - 1, cj, cj + 1):
                for (px, py, pr) in grid.get((a, b), ()):
                    if (px - x) ** 2 + (py - y) ** 2 < (pr + r) ** 2:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            placed.append((x, y, r))
            grid.setdefault((ci, cj), []).append((x, y, r))
    p = Particles(2)
    p.add_segment((0.0, 0.0), (W, 0.0))
    vel = (2.0 * splitmix_uniform(seed + 0x5851F42D, 2 * len(placed)).reshape(-1, 2) - 1.0) * vmax
    for k, (x, y, r) in enumerate(placed):
        m = (r / 0.01) ** 2
        prop = Property(mass=m, moment_inertia=0.5 * m * r * r, force=(0.0, -9.81 * m))
        if vmax > 0.0:
            prop.velocity = (float(vel[k, 0]), float(vel[k, 1]))
        p.add_sphere((x, y), r, prop)
    return p.finalize()


def pile_scenes(n_scenes: int = 256, seed: int = 4, nmin: int = 200, nmax: int = 5000, vmax: float = 0.0):
    """The batched workload: scene s is pile_scene(seed * 1000 + s)."""
    return [pile_scene(seed * 1000 + s, nmin, nmax, vmax) for s in range(n_scenes)]


# solver settings per workload (dmax, dt, tolerance, max_ite, vap)
SETTINGS = {
    "disks_2d": dict(dmax=0.01, dt=0.005, tolerance=1e-6, max_ite=40000, vap=0, steps=200),
    "box_3d": dict(dmax=0.0045, dt=1e-3, tolerance=1e-6, max_ite=40000, vap=1, steps=500),
    "spheres_1m": dict(dmax=0.0018, dt=1e-3, tolerance=1e-6, max_ite=40000, vap=0, steps=100),
    "pile_scenes": dict(dmax=0.009, dt=1e-3, tolerance=1e-6, max_ite=40000, vap=1, steps=1000),
    "se_pile": dict(dmax=0.004, dt=5e-4, tolerance=1e-6, max_ite=40000, vap=1, steps=300, mu=0.3),
}
