"""Python mirror of ``ScopiSolver<dim, problem, OptimGradient<apgd>, contact, vap>`` on the GPU.

Same names and meaning as the reference (include/scopi/solver.hpp:91-206):
``run(dt, total_it, initial_iter=0)``, ``current_contacts()``, ``get_params()`` with the
``optim_params`` (alpha, max_ite, tolerance, dynamic_descent), ``contact_method_params``
(dmax, kd_tree_radius), ``default_contact_property`` (mu, gamma, gamma_min, gamma_tol)
groups, and ``lagrange_multiplier()`` (OptimGradient.hpp:323-326).  Every call goes
through the C ABI of libscopi_gpu.so; the particles live on the GPU between calls.
Errors raise ``ScopiGPUError``; APGD non-convergence is reported like the reference
("APGD didn't converge." on stderr) and in ``stats()``.
"""
from __future__ import annotations

import ctypes as C
import sys
from types import SimpleNamespace

import numpy as np

from . import _abi
from ._abi import (BRUTE_FORCE, FP64, FRICTION, FRICTION_FIXED_POINT, KDTREE, MIXED, NOFRICTION,  # noqa: F401
                   VAP_FIXED, VAP_FPD, VISCOUS, VISCOUS_FRICTION)
from .container import ParticleArrays


class ScopiGPUError(RuntimeError):
    pass


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i64(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


class _ParamGroup(SimpleNamespace):
    pass


def _set_param(p, k, v):
    """One field of scopi_gpu_params; booleans and the box's 3-vectors converted."""
    if k == "dynamic_descent":
        v = 1 if v else 0
    elif k in ("box_lower", "box_upper"):
        v = (C.c_double * 3)(*([float(x) for x in v] + [0.0] * (3 - len(v))))
    elif k == "periodic":
        v = (C.c_int32 * 3)(*([int(bool(x)) for x in v] + [0] * (3 - len(v))))
    setattr(p, k, v)


class ScopiSolver:
    """GPU ScopiSolver.  ``particles`` is a ``ParticleArrays`` (obstacles first)."""

    def __init__(self, particles: ParticleArrays, problem=NOFRICTION, vap=VAP_FIXED, contact_method=KDTREE,
                 precision=FP64, device=0, **overrides):
        self._lib = _abi.load()
        p = _abi.Params()
        self._lib.scopi_gpu_default_params(C.byref(p), particles.dim)
        p.problem, p.vap, p.contact_method, p.precision, p.device = problem, vap, contact_method, precision, device
        for k, v in overrides.items():
            _set_param(p, k, v)
        self._params = p
        self._h = None
        self.particles = particles.copy()
        self._created = False

    # --- reference-style parameter access --------------------------------
    def get_params(self):
        p = self._params
        return SimpleNamespace(
            optim_params=_ParamGroup(alpha=p.alpha, max_ite=p.max_ite, tolerance=p.tolerance,
                                     dynamic_descent=bool(p.dynamic_descent)),
            contact_method_params=_ParamGroup(dmax=p.dmax, kd_tree_radius=p.kd_tree_radius),
            default_contact_property=_ParamGroup(mu=p.mu, gamma=p.gamma, gamma_min=p.gamma_min, gamma_tol=p.gamma_tol,
                                                 fixed_point_tol=p.fixed_point_tol,
                                                 fixed_point_max_iter=p.fixed_point_max_iter),
        )

    def set_params(self, **kw):
        if self._created:
            raise ScopiGPUError("parameters are fixed once the solver has run")
        for k, v in kw.items():
            setattr(self._params, k, v)

    # --- lifecycle --------------------------------------------------------
    def _check(self, rc, what):
        if rc < 0:
            msg = self._lib.scopi_gpu_last_error(self._h).decode()
            raise ScopiGPUError(f"{what} failed ({rc}): {msg}")
        return rc

    def _ensure(self):
        if self._created:
            return
        h = C.c_void_p()
        rc = self._lib.scopi_gpu_create(C.byref(self._params), C.byref(h))
        if rc < 0:
            raise ScopiGPUError(f"scopi_gpu_create failed ({rc}): {self._lib.scopi_gpu_last_error(None).decode()}")
        self._h = h
        self._created = True
        self._upload()

    def _struct(self, pa):
        self._keep = pa
        return _abi.ParticlesC(pa.n, pa.nb_inactive, pa.shape.ctypes.data_as(C.POINTER(C.c_int32)), _dp(pa.pos),
                               _dp(pa.q), _dp(pa.v), _dp(pa.omega), _dp(pa.vd), _dp(pa.omega_d), _dp(pa.f), _dp(pa.m),
                               _dp(pa.j), _dp(pa.radius), _dp(pa.length), _dp(pa.axes), _dp(pa.squareness),
                               pa.worm.ctypes.data_as(C.POINTER(C.c_int32)))

    def _upload(self):
        s = self._struct(self.particles)
        self._check(self._lib.scopi_gpu_set_particles(self._h, C.byref(s)), "scopi_gpu_set_particles")

    def set_particles(self, pa: ParticleArrays):
        """Replace the particle state (contacts of the last step are kept, as in the reference)."""
        self.particles = pa.copy()
        if self._created:
            self._upload()

    def sync(self) -> ParticleArrays:
        s = self._struct(self.particles)
        self._check(self._lib.scopi_gpu_get_particles(self._h, C.byref(s)), "scopi_gpu_get_particles")
        return self.particles

    def close(self):
        if self._created and self._h:
            self._lib.scopi_gpu_destroy(self._h)
        self._h = None
        self._created = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- the reference API ------------------------------------------------
    def run(self, dt: float, total_it: int, initial_iter: int = 0):
        self._ensure()
        rc = self._check(self._lib.scopi_gpu_run(self._h, dt, total_it, initial_iter), "scopi_gpu_run")
        if rc == _abi.ENOCONV:
            print("APGD didn't converge.", file=sys.stderr)
        self.sync()
        return self

    def detect(self):
        """contact_base::run on the current state; returns the sorted contact list."""
        self._ensure()
        n = C.c_int64()
        self._check(self._lib.scopi_gpu_detect(self._h, C.byref(n)), "scopi_gpu_detect")
        return self.current_contacts()

    def current_contacts(self):
        self._ensure()
        n = C.c_int64()
        self._check(self._lib.scopi_gpu_get_contacts(self._h, 0, C.byref(n), None, None, None, None, None, None, None),
                    "scopi_gpu_get_contacts")
        k = n.value
        ci = np.zeros(k, np.int64)
        cj = np.zeros(k, np.int64)
        d = np.zeros(k)
        g = np.zeros(k)
        nij = np.zeros((k, 3))
        pi = np.zeros((k, 3))
        pj = np.zeros((k, 3))
        self._check(self._lib.scopi_gpu_get_contacts(self._h, k, C.byref(n), _i64(ci), _i64(cj), _dp(d), _dp(nij),
                                                     _dp(pi), _dp(pj), _dp(g)), "scopi_gpu_get_contacts")
        return {"i": ci, "j": cj, "dij": d, "nij": nij, "pi": pi, "pj": pj, "gamma": g}

    def lagrange_multiplier(self):
        n = C.c_int64()
        self._check(self._lib.scopi_gpu_get_lambda(self._h, 0, C.byref(n), None), "scopi_gpu_get_lambda")
        out = np.zeros(n.value)
        self._check(self._lib.scopi_gpu_get_lambda(self._h, n.value, C.byref(n), _dp(out)), "scopi_gpu_get_lambda")
        return out

    def stats(self):
        s = _abi.Stats()
        self._check(self._lib.scopi_gpu_get_stats(self._h, C.byref(s)), "scopi_gpu_get_stats")
        return {k: getattr(s, k) for k, _ in _abi.Stats._fields_}

    def stream_handle(self) -> int:
        """The engine's cudaStream_t (as an int) for CUDA-event timing on that stream."""
        self._ensure()
        return int(self._lib.scopi_gpu_get_stream(self._h) or 0)

    def upload(self, pa: ParticleArrays):
        """Copy a full particle state from host arrays (scopi_gpu_set_particles)."""
        self._ensure()
        s = self._struct(pa)
        self._check(self._lib.scopi_gpu_set_particles(self._h, C.byref(s)), "scopi_gpu_set_particles")

    def upload_state(self, pa: ParticleArrays):
        """Copy pos/q/v/omega from host arrays into the container on the device
        (scopi_gpu_set_state); pa must hold as many bodies and obstacles as the device's
        container, and its other fields are not read."""
        self._ensure()
        s = self._struct(pa)
        self._check(self._lib.scopi_gpu_set_state(self._h, C.byref(s)), "scopi_gpu_set_state")

    def download(self, pa: ParticleArrays):
        """Copy pos/q/v/omega back into host arrays (scopi_gpu_get_particles)."""
        s = self._struct(pa)
        self._check(self._lib.scopi_gpu_get_particles(self._h, C.byref(s)), "scopi_gpu_get_particles")
        return pa

    def step(self, dt: float, n: int = 1) -> int:
        """n time steps without copying the particles back (device-resident state)."""
        self._ensure()
        return self._check(self._lib.scopi_gpu_run(self._h, dt, n, 0), "scopi_gpu_run")

    def kernel_launches(self) -> int:
        return int(self._lib.scopi_gpu_kernel_launches(self._h)) if self._h else 0

    def amat(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros(3 * len(self.current_contacts()["i"]))
        self._check(self._lib.scopi_gpu_amat(self._h, _dp(u), _dp(out)), "scopi_gpu_amat")
        return out

    def atmat(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros(6 * (self.particles.n - self.particles.nb_inactive))
        self._check(self._lib.scopi_gpu_atmat(self._h, _dp(f), _dp(out)), "scopi_gpu_atmat")
        return out


class ScopiBatch:
    """Many independent scenes stepped together (one ScopiSolver per scene in the reference).

    ``scenes`` is a list of ``ParticleArrays`` (each obstacles first).  ``run(dt, k)`` advances
    every scene k steps (one CUDA graph replay per step, one persistent launch solving every
    scene); ``scene(s)`` returns scene s's particles and ``scene_stats(s)`` its solver
    statistics of the last step.  ``problem``: NOFRICTION (FP64 or MIXED), FRICTION (FP64,
    ``mu`` in the overrides) or VISCOUS (FP64).  ``block_threads`` pins the threads per scene of the NoFriction
    solve (256, 512, 1024, or 2048: the largest scenes on two CTAs); 0 lets the first step
    autotune it.
    """

    def __init__(self, scenes, vap=VAP_FPD, contact_method=KDTREE, precision=FP64, device=0, block_threads=0,
                 tile=0, problem=NOFRICTION, **overrides):
        self._lib = _abi.load()
        p = _abi.Params()
        self._lib.scopi_gpu_default_params(C.byref(p), scenes[0].dim)
        p.problem, p.vap, p.contact_method, p.precision, p.device = problem, vap, contact_method, precision, device
        for k, v in overrides.items():
            _set_param(p, k, v)
        self._params = p
        self.scenes = [s.copy() for s in scenes]
        arr = (_abi.ParticlesC * len(self.scenes))()
        self._keep = []
        for k, pa in enumerate(self.scenes):
            arr[k] = _abi.ParticlesC(pa.n, pa.nb_inactive, pa.shape.ctypes.data_as(C.POINTER(C.c_int32)), _dp(pa.pos),
                                     _dp(pa.q), _dp(pa.v), _dp(pa.omega), _dp(pa.vd), _dp(pa.omega_d), _dp(pa.f),
                                     _dp(pa.m), _dp(pa.j), _dp(pa.radius), _dp(pa.length))
        h = C.c_void_p()
        rc = self._lib.scopi_gpu_batch_create(C.byref(p), len(self.scenes), arr, C.byref(h))
        if rc < 0:
            raise ScopiGPUError(f"scopi_gpu_batch_create failed ({rc}): {self._lib.scopi_gpu_last_error(None).decode()}")
        self._h = h
        if block_threads and tile:
            self._check(self._lib.scopi_gpu_batch_set_shape(h, int(block_threads), int(tile)),
                        "scopi_gpu_batch_set_shape")
        elif block_threads:
            self._check(self._lib.scopi_gpu_batch_set_block_threads(h, int(block_threads)),
                        "scopi_gpu_batch_set_block_threads")

    def _check(self, rc, what):
        if rc < 0:
            raise ScopiGPUError(f"{what} failed ({rc}): {self._lib.scopi_gpu_last_error(self._h).decode()}")
        return rc

    def run(self, dt: float, steps: int):
        rc = self._check(self._lib.scopi_gpu_run(self._h, dt, steps, 0), "scopi_gpu_run")
        if rc == _abi.ENOCONV:
            print("APGD didn't converge.", file=sys.stderr)
        return self

    def scene(self, s: int) -> ParticleArrays:
        pa = self.scenes[s]
        st = _abi.ParticlesC(pa.n, pa.nb_inactive, pa.shape.ctypes.data_as(C.POINTER(C.c_int32)), _dp(pa.pos), _dp(pa.q),
                             _dp(pa.v), _dp(pa.omega), _dp(pa.vd), _dp(pa.omega_d), _dp(pa.f), _dp(pa.m), _dp(pa.j),
                             _dp(pa.radius), _dp(pa.length))
        self._check(self._lib.scopi_gpu_batch_get_scene(self._h, s, C.byref(st)), "scopi_gpu_batch_get_scene")
        return pa

    def scene_stats(self, s: int):
        st = _abi.SceneStats()
        self._check(self._lib.scopi_gpu_batch_get_scene_stats(self._h, s, C.byref(st)), "scopi_gpu_batch_get_scene_stats")
        return {k: getattr(st, k) for k, _ in _abi.SceneStats._fields_}

    def stats(self):
        s = _abi.Stats()
        self._check(self._lib.scopi_gpu_get_stats(self._h, C.byref(s)), "scopi_gpu_get_stats")
        return {k: getattr(s, k) for k, _ in _abi.Stats._fields_}

    def block_threads(self) -> int:
        return int(self._lib.scopi_gpu_batch_block_threads(self._h))

    def tile(self) -> int:
        """Contacts each thread of the batched solve keeps in flight (autotuned with block_threads)."""
        return int(self._lib.scopi_gpu_batch_tile(self._h))

    def stream_handle(self) -> int:
        return int(self._lib.scopi_gpu_get_stream(self._h) or 0)

    def kernel_launches(self) -> int:
        return int(self._lib.scopi_gpu_kernel_launches(self._h))

    def close(self):
        if self._h:
            self._lib.scopi_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
