"""ctypes view of the C ABI declared in include/scopi_gpu.h (libscopi_gpu.so, sm_100a).

The library is built in-tree (scopi_b200/build.py).  There is no fallback: if the
shared library is missing or cannot be loaded, importing the solver raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscopi_gpu.so")

OK, EINVAL, ECUDA, ENOMEM, EUNSUPPORTED, ETIMEOUT, ENOCONV = 0, -1, -2, -3, -4, -5, 1
NOFRICTION, FRICTION, VISCOUS, FRICTION_FIXED_POINT, VISCOUS_FRICTION = 0, 1, 2, 3, 4
VAP_FIXED, VAP_FPD = 0, 1
BRUTE_FORCE, KDTREE = 0, 1
FP64, MIXED = 0, 1

EXPORTED = [
    "scopi_gpu_default_params", "scopi_gpu_create", "scopi_gpu_destroy", "scopi_gpu_set_particles",
    "scopi_gpu_get_particles", "scopi_gpu_run", "scopi_gpu_detect", "scopi_gpu_get_contacts",
    "scopi_gpu_get_lambda", "scopi_gpu_get_stats", "scopi_gpu_amat", "scopi_gpu_atmat",
    "scopi_gpu_last_error", "scopi_gpu_kernel_launches", "scopi_gpu_get_stream", "scopi_gpu_apgd_noalloc",
    "scopi_gpu_batch_create", "scopi_gpu_batch_get_scene", "scopi_gpu_batch_get_scene_stats",
    "scopi_gpu_batch_block_threads", "scopi_gpu_batch_set_block_threads", "scopi_gpu_test_barrier_stall",
    "scopi_gpu_set_contacts", "scopi_gpu_get_se_starts", "scopi_gpu_batch_tile", "scopi_gpu_batch_set_shape",
    "scopi_gpu_set_state",
]


class Params(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("problem", C.c_int32), ("vap", C.c_int32), ("contact_method", C.c_int32),
        ("precision", C.c_int32), ("dynamic_descent", C.c_int32), ("max_ite", C.c_int64), ("dmax", C.c_double),
        ("kd_tree_radius", C.c_double), ("alpha", C.c_double), ("tolerance", C.c_double), ("mu", C.c_double),
        ("gamma", C.c_double), ("gamma_min", C.c_double), ("gamma_tol", C.c_double),
        ("mixed_violation_tol", C.c_double), ("mixed_max_corrections", C.c_int32), ("device", C.c_int32),
        ("initial_step", C.c_int32), ("fixed_point_tol", C.c_double), ("fixed_point_max_iter", C.c_int64),
        ("box_lower", C.c_double * 3), ("box_upper", C.c_double * 3), ("periodic", C.c_int32 * 3),
        ("barrier_timeout_us", C.c_int32),
    ]


class ParticlesC(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("nb_inactive", C.c_int64), ("shape", C.POINTER(C.c_int32)),
        ("pos", C.POINTER(C.c_double)), ("q", C.POINTER(C.c_double)), ("v", C.POINTER(C.c_double)),
        ("omega", C.POINTER(C.c_double)), ("vd", C.POINTER(C.c_double)), ("omega_d", C.POINTER(C.c_double)),
        ("f", C.POINTER(C.c_double)), ("m", C.POINTER(C.c_double)), ("j", C.POINTER(C.c_double)),
        ("radius", C.POINTER(C.c_double)), ("length", C.POINTER(C.c_double)),
        ("axes", C.POINTER(C.c_double)), ("squareness", C.POINTER(C.c_double)), ("worm", C.POINTER(C.c_int32)),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("contacts", C.c_int64), ("iterations", C.c_int64), ("backtracks", C.c_int64), ("restarts", C.c_int64),
        ("fp32_iterations", C.c_int64), ("corrections", C.c_int64), ("converged", C.c_int32),
        ("status", C.c_int32), ("violation", C.c_double), ("ms_step", C.c_double), ("ms_solve", C.c_double),
        ("ms_apgd_kernel", C.c_double), ("steps", C.c_int64), ("fixed_point_iterations", C.c_int64),
    ]


class SceneStats(C.Structure):
    _fields_ = [
        ("contacts", C.c_int64), ("iterations", C.c_int64), ("fp32_iterations", C.c_int64), ("backtracks", C.c_int64),
        ("restarts", C.c_int64), ("corrections", C.c_int32), ("converged", C.c_int32), ("violation", C.c_double),
    ]


_lib = None


def load(path: str = LIB_PATH):
    """Load libscopi_gpu.so and declare its signatures.  Raises OSError if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with `python -m scopi_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(path)
    H = C.c_void_p
    D = C.POINTER(C.c_double)
    I64 = C.POINTER(C.c_int64)
    L.scopi_gpu_default_params.argtypes = [C.POINTER(Params), C.c_int32]
    L.scopi_gpu_default_params.restype = None
    L.scopi_gpu_create.argtypes = [C.POINTER(Params), C.POINTER(H)]
    L.scopi_gpu_destroy.argtypes = [H]
    L.scopi_gpu_set_particles.argtypes = [H, C.POINTER(ParticlesC)]
    L.scopi_gpu_get_particles.argtypes = [H, C.POINTER(ParticlesC)]
    L.scopi_gpu_set_state.argtypes = [H, C.POINTER(ParticlesC)]
    L.scopi_gpu_run.argtypes = [H, C.c_double, C.c_int64, C.c_int64]
    L.scopi_gpu_detect.argtypes = [H, I64]
    L.scopi_gpu_get_contacts.argtypes = [H, C.c_int64, I64, I64, I64, D, D, D, D, D]
    L.scopi_gpu_get_lambda.argtypes = [H, C.c_int64, I64, D]
    L.scopi_gpu_get_stats.argtypes = [H, C.POINTER(Stats)]
    L.scopi_gpu_amat.argtypes = [H, D, D]
    L.scopi_gpu_atmat.argtypes = [H, D, D]
    L.scopi_gpu_last_error.argtypes = [H]
    L.scopi_gpu_last_error.restype = C.c_char_p
    L.scopi_gpu_kernel_launches.argtypes = [H]
    L.scopi_gpu_kernel_launches.restype = C.c_int64
    L.scopi_gpu_get_stream.argtypes = [H]
    L.scopi_gpu_get_stream.restype = C.c_void_p
    P = C.c_void_p  # device pointers
    L.scopi_gpu_apgd_noalloc.argtypes = [C.c_int32, C.c_int64, C.c_int64, C.c_int64, P, P, P, P, P, P, P, C.c_double,
                                         C.c_double, C.c_double, C.c_int64, C.c_int32, P, P, I64, C.c_void_p]
    L.scopi_gpu_apgd_noalloc.restype = C.c_int32
    L.scopi_gpu_batch_create.argtypes = [C.POINTER(Params), C.c_int32, C.POINTER(ParticlesC), C.POINTER(H)]
    L.scopi_gpu_batch_create.restype = C.c_int32
    L.scopi_gpu_batch_get_scene.argtypes = [H, C.c_int32, C.POINTER(ParticlesC)]
    L.scopi_gpu_batch_get_scene.restype = C.c_int32
    L.scopi_gpu_batch_get_scene_stats.argtypes = [H, C.c_int32, C.POINTER(SceneStats)]
    L.scopi_gpu_batch_get_scene_stats.restype = C.c_int32
    L.scopi_gpu_batch_block_threads.argtypes = [H]
    L.scopi_gpu_batch_block_threads.restype = C.c_int32
    L.scopi_gpu_batch_set_block_threads.argtypes = [H, C.c_int32]
    L.scopi_gpu_batch_set_block_threads.restype = C.c_int32
    L.scopi_gpu_get_se_starts.argtypes = [H, C.c_int64, I64, D]
    L.scopi_gpu_get_se_starts.restype = C.c_int32
    L.scopi_gpu_set_contacts.argtypes = [H, C.c_int64, I64, I64, D, D, D, D]
    L.scopi_gpu_set_contacts.restype = C.c_int32
    L.scopi_gpu_batch_tile.argtypes = [H]
    L.scopi_gpu_batch_tile.restype = C.c_int32
    L.scopi_gpu_batch_set_shape.argtypes = [H, C.c_int32, C.c_int32]
    L.scopi_gpu_batch_set_shape.restype = C.c_int32
    L.scopi_gpu_test_barrier_stall.argtypes = [H]
    L.scopi_gpu_test_barrier_stall.restype = C.c_int32
    for name in ("scopi_gpu_create", "scopi_gpu_destroy", "scopi_gpu_set_particles", "scopi_gpu_get_particles",
                 "scopi_gpu_set_state",
                 "scopi_gpu_run", "scopi_gpu_detect", "scopi_gpu_get_contacts", "scopi_gpu_get_lambda",
                 "scopi_gpu_get_stats", "scopi_gpu_amat", "scopi_gpu_atmat"):
        getattr(L, name).restype = C.c_int32
    _lib = L
    return L
