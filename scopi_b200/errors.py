"""Error of one contact solve against another on the same contacts, evaluated on the host in FP64.

Used to state the mixed form's error against the FP64 form (same state, same contact list):
multipliers lambda, post-solve velocities v and post-solve gaps

    gap_c = d_c + dt n_c . (v_i - v_j)

(the first-order distance the step leaves between the two bodies; obstacles do not enter
the contact Jacobian, matrix/velocities.hpp:67-144 of the reference, so their velocity counts
as zero).  The negative part of the gap is the constraint violation the solver reports.

Also the optimality test of a normal-contact (NoFriction) solve at any size: with
u = M^-1 B^T lambda and v = U + dt u (U the a-priori velocities), lambda >= 0, gap >= 0 and
gap_c = 0 wherever lambda_c > 0 are the KKT conditions of the QP the reference's APGD
solves (minimization_problem.hpp:122-134); `normal_kkt` measures each of them.
"""
from __future__ import annotations

import numpy as np


def step_gaps(contacts, v, dt, nb_inactive):
    """gap_c = d_c + dt n_c.(v_i - v_j) with v of obstacles taken as 0."""
    vv = np.array(v, dtype=np.float64, copy=True)
    vv[:nb_inactive] = 0.0
    i, j = contacts["i"], contacts["j"]
    n = contacts["nij"]
    return contacts["dij"] + dt * np.einsum("cd,cd->c", n, vv[i] - vv[j])


def _rel(a, b):
    den = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def solve_errors(ref, other, dt, nb_inactive):
    """ref / other: dicts with 'contacts', 'lambda', 'v' (all bodies) of two solves of the
    same step.  Returns relative (2-norm) and max-abs errors of lambda, v and the gaps."""
    cr, co = ref["contacts"], other["contacts"]
    if not (np.array_equal(cr["i"], co["i"]) and np.array_equal(cr["j"], co["j"])):
        raise ValueError("the two solves have different contact lists")
    lr, lo = np.asarray(ref["lambda"]), np.asarray(other["lambda"])
    vr = np.asarray(ref["v"])[nb_inactive:]
    vo = np.asarray(other["v"])[nb_inactive:]
    gr = step_gaps(cr, ref["v"], dt, nb_inactive)
    go = step_gaps(co, other["v"], dt, nb_inactive)
    return {
        "contacts": int(len(cr["i"])),
        "lambda_rel": _rel(lo, lr), "lambda_max_abs": float(np.max(np.abs(lo - lr))) if len(lr) else 0.0,
        "lambda_max": float(np.max(np.abs(lr))) if len(lr) else 0.0,
        "v_rel": _rel(vo, vr), "v_max_abs": float(np.max(np.abs(vo - vr))) if len(vr) else 0.0,
        "gap_max_abs": float(np.max(np.abs(go - gr))) if len(gr) else 0.0,
        "violation_ref": float(max(0.0, -np.min(gr))) if len(gr) else 0.0,
        "violation_other": float(max(0.0, -np.min(go))) if len(go) else 0.0,
    }


def normal_kkt(contacts, lam, v_after, U, inv_mass, dt, nb_inactive):
    """Optimality of a NoFriction solve: lam (one per contact), v_after (all bodies, the
    solver's velocities), U (a-priori velocities of all bodies), inv_mass (active bodies).

    Returns: v_consistency = |v_after - (U + dt M^-1 B^T lam)| / |v_after| over the active
    bodies; lambda_min; violation = max(0, -min gap); stationarity = max |gap_c| over the
    contacts with lam_c > 1e-6 max(lam); complementarity = max |lam_c gap_c|."""
    nin = nb_inactive
    i, j, n = contacts["i"], contacts["j"], contacts["nij"]
    na = len(inv_mass)
    w = np.zeros((na, 3))
    for d in range(3):
        f = lam * n[:, d]
        ai = i >= nin
        aj = j >= nin
        w[:, d] += np.bincount(i[ai] - nin, weights=f[ai], minlength=na)
        w[:, d] -= np.bincount(j[aj] - nin, weights=f[aj], minlength=na)
    v_exp = np.array(U, dtype=np.float64, copy=True)
    v_exp[nin:] += dt * w * np.asarray(inv_mass)[:, None]
    va = np.asarray(v_after)[nin:]
    cons = float(np.linalg.norm(va - v_exp[nin:]) / max(np.linalg.norm(va), 1e-300))
    g = step_gaps(contacts, v_exp, dt, nin)
    big = lam > 1e-6 * float(np.max(lam)) if len(lam) else np.zeros(0, bool)
    return {
        "v_consistency": cons,
        "lambda_min": float(np.min(lam)) if len(lam) else 0.0,
        "violation": float(max(0.0, -np.min(g))) if len(g) else 0.0,
        "stationarity": float(np.max(np.abs(g[big]))) if np.any(big) else 0.0,
        "complementarity": float(np.max(np.abs(lam * g))) if len(g) else 0.0,
        "active": int(np.count_nonzero(big)),
    }
