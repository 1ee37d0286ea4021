"""scopi_b200 -- B200 (sm_100a) engine for the SCoPI contact-dynamics time step.

The compute path is libscopi_gpu.so (CUDA, C ABI in include/scopi_gpu.h).  This
package holds the host-side mirror of the reference's interface (ScopiSolver,
particle container) and seeded synthetic workloads.
"""
from .container import PLANE, SEGMENT, SPHERE, ParticleArrays, Particles, Property, quaternion  # noqa: F401
from .solver import (BRUTE_FORCE, FP64, FRICTION, FRICTION_FIXED_POINT, KDTREE, MIXED, NOFRICTION,  # noqa: F401
                     VAP_FIXED, VAP_FPD, VISCOUS, VISCOUS_FRICTION, ScopiBatch, ScopiGPUError, ScopiSolver)
