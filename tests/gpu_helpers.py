"""Shared helpers of the GPU parity tests (oracle vs libscopi_gpu on the same inputs)."""
import numpy as np

import py_oracle as orc
from scopi_b200 import ScopiSolver
from scopi_b200.container import Particles, Property


def gpu_solver(pa, **kw):
    kw = dict(kw)
    prec = kw.pop("precision", 0)
    problem = kw.pop("problem", 0)
    vap = kw.pop("vap", 0)
    method = kw.pop("contact_method", 1)
    return ScopiSolver(pa, problem=problem, vap=vap, contact_method=method, precision=prec, **kw)


def oracle_solver(pa, **kw):
    kw = dict(kw)
    kw.pop("precision", None)
    return orc.OracleSolver(pa, **kw)


def same_contacts(a, b):
    """(i, j) lists equal and geometry bitwise equal."""
    assert np.array_equal(a["i"], b["i"]) and np.array_equal(a["j"], b["j"]), "contact pairs differ"
    for k in ("dij", "nij", "pi", "pj"):
        assert np.array_equal(a[k], b[k]), f"{k} differs (max {np.max(np.abs(a[k] - b[k]))})"


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.linalg.norm(b), 1e-300)
    return float(np.linalg.norm(a - b) / den)


def segment_pile(n=40, seed=3):
    """2D disks above a segment obstacle (the pile-of-sand setting), some within dmax."""
    rng = np.random.default_rng(seed)
    p = Particles(2)
    p.add_segment((0.0, 0.0), (0.6, 0.0))
    placed = []
    while len(placed) < n:
        r = rng.uniform(0.008, 0.012)
        x = rng.uniform(-0.05, 0.65)
        y = rng.uniform(0.005, 0.25)
        if all((x - a) ** 2 + (y - b) ** 2 > (r + c + 0.001) ** 2 for a, b, c in placed):
            placed.append((x, y, r))
    for x, y, r in placed:
        m = (r / 0.01) ** 2
        p.add_sphere((x, y), r, Property(mass=m, moment_inertia=0.5 * m * r * r, force=(0.0, -9.81 * m)))
    return p.finalize()
