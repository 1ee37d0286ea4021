"""Host-side particle container mirroring the reference's data model.

Mirrors ``scopi_container<dim>`` / ``property<dim>`` (include/scopi/container.hpp:339-384,
include/scopi/property.hpp:16-200) and the shape constructors the hot path uses:
``sphere`` (objects/types/sphere.hpp), ``plane`` (objects/types/plane.hpp:50-70),
``segment`` (objects/types/segment.hpp:133-138) and ``superellipsoid``
(objects/types/superellipsoid.hpp:59-70: centre, rotation, semi-axes, squareness (e, n)).

Layout (shared with the C-ABI ``scopi_gpu_particles`` in include/scopi_gpu.h):
every vector quantity has 3 slots per body.  In 2D the z slot of pos, v, vd and f
is 0 and the scalar rotation quantities (omega, desired omega, moment of inertia)
are stored in the z slot.  Quaternions are (w, x, y, z).  Obstacles (inactive
bodies) must be pushed before active particles, as in the reference
(container.hpp:365-373), which raises otherwise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SPHERE, PLANE, SEGMENT, SUPERELLIPSOID = 0, 1, 2, 3


def quaternion(angle: float, axes=(0.0, 0.0, 1.0)) -> np.ndarray:
    """``scopi::quaternion(angle, axes)`` (src/quaternion.cpp:12-36): normalised (cos a/2, sin a/2 * axes).

    A 2-component axis gets z = 1 appended, as the reference does.
    """
    ax = list(axes)
    if len(ax) == 2:
        ax = [ax[0], ax[1], 1.0]
    s = math.sin(angle / 2)
    out = np.array([math.cos(angle / 2), s * ax[0], s * ax[1], s * ax[2]], dtype=np.float64)
    nrm = math.sqrt(float(out[0] * out[0] + out[1] * out[1] + out[2] * out[2] + out[3] * out[3]))
    return out / nrm


@dataclass
class Property:
    """``scopi::property<dim>`` builder values (property.hpp:16-200)."""

    velocity: tuple = (0.0, 0.0, 0.0)
    desired_velocity: tuple = (0.0, 0.0, 0.0)
    omega: object = 0.0
    desired_omega: object = 0.0
    force: tuple = (0.0, 0.0, 0.0)
    mass: float = 1.0
    moment_inertia: object = 0.0
    active: bool = True

    def deactivate(self) -> "Property":
        self.active = False
        return self


def _vec3(x, dim):
    a = np.zeros(3)
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    a[: min(len(x), dim)] = x[: min(len(x), dim)]
    return a


def _rot3(x, dim):
    """Rotation quantity: scalar in 2D (stored in z), 3-vector in 3D."""
    a = np.zeros(3)
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    if dim == 2:
        a[2] = x[0] if len(x) == 1 else x[-1]
    else:
        a[:] = x if len(x) == 3 else x[0]
    return a


@dataclass
class Particles:
    """Structure-of-arrays particle store (obstacles first)."""

    dim: int
    shape: list = field(default_factory=list)
    pos: list = field(default_factory=list)
    q: list = field(default_factory=list)
    v: list = field(default_factory=list)
    omega: list = field(default_factory=list)
    vd: list = field(default_factory=list)
    omega_d: list = field(default_factory=list)
    f: list = field(default_factory=list)
    m: list = field(default_factory=list)
    j: list = field(default_factory=list)
    radius: list = field(default_factory=list)
    length: list = field(default_factory=list)
    axes: list = field(default_factory=list)
    squareness: list = field(default_factory=list)
    worm: list = field(default_factory=list)
    nb_inactive: int = 0
    n_worms: int = 0

    # --- builders --------------------------------------------------------
    def _push(self, shape, pos, q, prop: Property, radius=0.0, length=0.0, axes=(0.0, 0.0, 0.0), squareness=(1.0, 1.0),
              worm=-1):
        n = len(self.shape)
        if not prop.active:
            if self.nb_inactive != n:
                raise RuntimeError("All the obstacles must be pushed before the active particles.")
            self.nb_inactive += 1
        self.shape.append(shape)
        self.pos.append(_vec3(pos, self.dim))
        self.q.append(np.asarray(q, dtype=np.float64))
        self.v.append(_vec3(prop.velocity, self.dim))
        self.vd.append(_vec3(prop.desired_velocity, self.dim))
        self.omega.append(_rot3(prop.omega, self.dim))
        self.omega_d.append(_rot3(prop.desired_omega, self.dim))
        self.f.append(_vec3(prop.force, self.dim))
        self.m.append(float(prop.mass))
        self.j.append(_rot3(prop.moment_inertia, self.dim))
        self.radius.append(float(radius))
        self.length.append(float(length))
        self.axes.append(np.asarray(axes, dtype=np.float64))
        self.squareness.append(np.asarray(squareness, dtype=np.float64))
        self.worm.append(int(worm))
        return self

    def add_sphere(self, pos, radius, prop: Property | None = None, q=None):
        q = quaternion(0.0) if q is None else q
        return self._push(SPHERE, pos, q, prop or Property(), radius=radius)

    def add_plane(self, pos, angle=0.0, prop: Property | None = None, q=None):
        """``plane<dim>(pos, angle)`` uses quaternion(angle) about z; ``q`` overrides it."""
        q = quaternion(angle) if q is None else q
        return self._push(PLANE, pos, q, prop or Property().deactivate())

    def add_segment(self, p1, p2, prop: Property | None = None):
        """``segment<2>(pos1, pos2)``: centre, quaternion(atan2(x1-x2, y2-y1)), length |p2-p1|."""
        p1 = np.asarray(p1, dtype=np.float64)
        p2 = np.asarray(p2, dtype=np.float64)
        ang = math.atan2(p1[0] - p2[0], p2[1] - p1[1])
        d = p2 - p1
        length = math.sqrt(float(np.dot(d, d)))
        return self._push(SEGMENT, 0.5 * (p1 + p2), quaternion(ang), prop or Property().deactivate(), length=length)

    def add_superellipsoid(self, pos, radius, squareness, prop: Property | None = None, q=None):
        """``superellipsoid<dim>(pos, q, radius, squareness)``: semi-axes (rx, ry, rz) and
        squareness (e, n) in 3D, (rx, ry) and e in 2D (superellipsoid.hpp:59-70; stored as
        (rx, ry, 0) and (e, 1)).  ``radius`` of the body record holds the bounding radius
        |semi-axes| (the body lies in its axis box for squareness <= 2), which the contact
        search uses; the closest points use the exact surface."""
        if self.dim == 3:
            r = np.asarray(radius, dtype=np.float64).reshape(3)
            sq = np.asarray(squareness, dtype=np.float64).reshape(2)
        else:
            r = np.concatenate([np.asarray(radius, dtype=np.float64).reshape(2), [0.0]])
            sq = np.array([float(np.asarray(squareness, dtype=np.float64).reshape(-1)[0]), 1.0])
        q = quaternion(0.0) if q is None else q
        return self._push(SUPERELLIPSOID, pos, q, prop or Property(), radius=float(np.sqrt(np.dot(r, r))), axes=r,
                          squareness=sq)

    def add_worm(self, positions, radius, prop: Property | None = None, q=None):
        """``worm<dim>(pos, q, radius, size)`` (objects/types/worm.hpp:118-131) pushed with one
        property (container.hpp:338-384): one sphere body per position, all of ``radius``,
        each with the property's values, tagged with the worm's index.  The solver glues
        consecutive spheres of a worm (add_contact.hpp:11-28)."""
        prop = prop or Property()
        if not prop.active:
            raise ValueError("worms are active objects")
        w = self.n_worms
        self.n_worms += 1
        qs = [quaternion(0.0)] * len(positions) if q is None else list(q)
        for pos, qq in zip(positions, qs):
            self._push(SPHERE, pos, qq, prop, radius=radius, worm=w)
        return self

    # --- array views -----------------------------------------------------
    def finalize(self) -> "ParticleArrays":
        return ParticleArrays.from_lists(self)


@dataclass
class ParticleArrays:
    """Contiguous numpy arrays in the C-ABI layout."""

    dim: int
    nb_inactive: int
    shape: np.ndarray
    pos: np.ndarray
    q: np.ndarray
    v: np.ndarray
    omega: np.ndarray
    vd: np.ndarray
    omega_d: np.ndarray
    f: np.ndarray
    m: np.ndarray
    j: np.ndarray
    radius: np.ndarray
    length: np.ndarray
    axes: np.ndarray = None        # n x 3 superellipsoid semi-axes (0 for other shapes)
    squareness: np.ndarray = None  # n x 2 superellipsoid squareness (e, n)
    worm: np.ndarray = None        # n int32: index of the worm a sphere belongs to, -1 if none

    def __post_init__(self):
        n = int(self.shape.shape[0])
        if self.axes is None:
            self.axes = np.zeros((n, 3))
        if self.squareness is None:
            self.squareness = np.ones((n, 2))
        self.axes = np.ascontiguousarray(self.axes, dtype=np.float64).reshape(n, 3)
        self.squareness = np.ascontiguousarray(self.squareness, dtype=np.float64).reshape(n, 2)
        if self.worm is None:
            self.worm = np.full(n, -1, np.int32)
        self.worm = np.ascontiguousarray(self.worm, dtype=np.int32).reshape(n)

    @property
    def n(self) -> int:
        return int(self.shape.shape[0])

    @staticmethod
    def from_lists(p: Particles) -> "ParticleArrays":
        def a2(x, w):
            return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, w))

        return ParticleArrays(
            dim=p.dim,
            nb_inactive=p.nb_inactive,
            shape=np.ascontiguousarray(np.asarray(p.shape, dtype=np.int32)),
            pos=a2(p.pos, 3), q=a2(p.q, 4), v=a2(p.v, 3), omega=a2(p.omega, 3),
            vd=a2(p.vd, 3), omega_d=a2(p.omega_d, 3), f=a2(p.f, 3),
            m=np.ascontiguousarray(np.asarray(p.m, dtype=np.float64)),
            j=a2(p.j, 3),
            radius=np.ascontiguousarray(np.asarray(p.radius, dtype=np.float64)),
            length=np.ascontiguousarray(np.asarray(p.length, dtype=np.float64)),
            axes=a2(p.axes, 3) if p.axes else None,
            squareness=a2(p.squareness, 2) if p.squareness else None,
            worm=np.ascontiguousarray(np.asarray(p.worm, dtype=np.int32)) if p.worm else None,
        )

    def copy(self) -> "ParticleArrays":
        return ParticleArrays(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})
