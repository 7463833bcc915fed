"""NumPy restatement of the reference Krylov solvers.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Each solver takes ``matvec`` / ``rmatvec`` callables on NumPy arrays and returns
a dict with the same fields as the reference ``SolverResult``
(``src/em3d/solvers/base.py:28-44``).  Scalars are cast to the vector dtype
where the reference casts them with ``be.complex_dtype``.
"""
from __future__ import annotations

import numpy as np


def _result(u, iterations, history, status, matvecs, rmatvecs, counts):
    return {
        "u": u,
        "iterations": int(iterations),
        "residual_history": [float(v) for v in history],
        "converged": status == "converged",
        "matvec_count": int(matvecs),
        "rmatvec_count": int(rmatvecs),
        "residual_action_counts": [int(c) for c in counts],
        "status": status,
        "true_final_residual": float(history[-1]) if history else float("inf"),
    }


def bicgstab(matvec, rhs, *, max_iter=200, rtol=1e-6, atol=0.0, divergence_guard=None,
             max_operator_actions=None):
    """Restates ``BiCGStab.solve`` (reference ``src/em3d/solvers/bicgstab.py:12-211``)."""
    cdt = rhs.dtype.type
    rhs_norm = float(np.linalg.norm(rhs))
    u = np.zeros_like(rhs)
    if rhs_norm == 0.0:
        return _result(u, 0, [0.0], "converged", 0, 0, [0])
    tol = max(float(rtol), float(atol) / rhs_norm)
    mv = 0
    hist, counts = [], []
    r = rhs - matvec(u)
    mv += 1
    rel0 = float(np.linalg.norm(r)) / rhs_norm
    hist.append(rel0)
    counts.append(mv)
    if not np.isfinite(rel0):
        return _result(u, 0, hist, "nonfinite", mv, 0, counts)
    if rel0 < tol:
        return _result(u, 0, hist, "converged", mv, 0, counts)
    if max_operator_actions is not None and mv >= int(max_operator_actions):
        return _result(u, 0, hist, "max_operator_actions", mv, 0, counts)

    r_hat = r.copy()
    rho_prev = 1.0 + 0.0j
    alpha = 1.0 + 0.0j
    omega = 1.0 + 0.0j
    v = np.zeros_like(rhs)
    p = np.zeros_like(rhs)
    status = "max_iter"
    done = 0
    budget = None if max_operator_actions is None else int(max_operator_actions)
    for it in range(int(max_iter)):
        rho = complex(np.vdot(r_hat, r))
        if abs(rho) == 0.0:
            status = "breakdown_rho"
            break
        if it == 0:
            p = r.copy()
        else:
            if abs(omega) == 0.0:
                status = "breakdown_omega"
                break
            beta = (rho / rho_prev) * (alpha / omega)
            p = r + cdt(beta) * (p - cdt(omega) * v)
        if budget is not None and mv + 1 > budget:
            status = "max_operator_actions"
            break
        v = matvec(p)
        mv += 1
        den = complex(np.vdot(r_hat, v))
        if abs(den) == 0.0:
            status = "breakdown_alpha"
            break
        alpha = rho / den
        s = r - cdt(alpha) * v
        s_rel = float(np.linalg.norm(s)) / rhs_norm
        u_alpha = u + cdt(alpha) * p

        def _stop(st):
            hist.append(s_rel)
            counts.append(mv)
            return st

        if not np.isfinite(s_rel):
            u, done, status = u_alpha, it + 1, _stop("nonfinite")
            break
        if divergence_guard is not None and s_rel > float(divergence_guard):
            u, done, status = u_alpha, it + 1, _stop("divergence_guard")
            break
        if s_rel < tol:
            u, done, status = u_alpha, it + 1, _stop("converged")
            break
        if budget is not None and mv + 1 > budget:
            u, done, status = u_alpha, it + 1, _stop("max_operator_actions")
            break
        t = matvec(s)
        mv += 1
        tt = complex(np.vdot(t, t))
        if abs(tt) < 1e-30 * rhs_norm * rhs_norm:
            u, done, status = u_alpha, it + 1, _stop("breakdown_t")
            break
        omega = complex(np.vdot(t, s)) / tt
        if abs(omega) == 0.0:
            u, done, status = u_alpha, it + 1, _stop("breakdown_omega")
            break
        u = u_alpha + cdt(omega) * s
        r = s - cdt(omega) * t
        done = it + 1
        rel = float(np.linalg.norm(r)) / rhs_norm
        hist.append(rel)
        counts.append(mv)
        if not np.isfinite(rel):
            status = "nonfinite"
            break
        if rel < tol:
            status = "converged"
            break
        if divergence_guard is not None and rel > float(divergence_guard):
            status = "divergence_guard"
            break
        rho_prev = rho
    else:
        status = "max_iter"
    return _result(u, done, hist, status, mv, 0, counts)


def sim(matvec, rhs, *, mu, max_iter=200, rtol=1e-6, atol=0.0, divergence_guard=None,
        max_operator_actions=None):
    """Restates ``SIM.solve`` (reference ``src/em3d/solvers/sim.py:13-91``)."""
    if mu is None or abs(mu) == 0.0:
        raise ValueError("SolverConfig: mu must be non-zero")
    cdt = rhs.dtype.type
    gamma = 1.0 / complex(mu)
    u = np.zeros_like(rhs)
    rhs_norm = float(np.linalg.norm(rhs))
    if rhs_norm == 0.0:
        return _result(u, 0, [0.0], "converged", 0, 0, [0])
    tol = max(float(rtol), float(atol) / rhs_norm)
    updates = mv = 0
    hist, counts = [], []
    while True:
        res = matvec(u) - rhs
        mv += 1
        rel = float(np.linalg.norm(res)) / rhs_norm
        hist.append(rel)
        counts.append(mv)
        if not np.isfinite(rel):
            status = "nonfinite"
            break
        if rel < tol:
            status = "converged"
            break
        if divergence_guard is not None and rel > float(divergence_guard):
            status = "divergence_guard"
            break
        if max_operator_actions is not None and mv >= int(max_operator_actions):
            status = "max_operator_actions"
            break
        if updates >= int(max_iter):
            status = "max_iter"
            break
        u = u - cdt(gamma) * res
        updates += 1
    return _result(u, updates, hist, status, mv, 0, counts)


def twostep(matvec, rmatvec, rhs, *, max_iter=200, rtol=1e-6, atol=0.0, divergence_guard=None,
            max_operator_actions=None):
    """Restates ``TwoStep.solve`` (reference ``src/em3d/solvers/twostep.py:16-139``)."""
    cdt = rhs.dtype.type

    def rdot(a, b):
        return float(np.vdot(a, b).real)

    rhs_norm = float(np.linalg.norm(rhs))
    u = np.zeros_like(rhs)
    if rhs_norm == 0.0:
        return _result(u, 0, [0.0], "converged", 0, 0, [0])
    tol = max(float(rtol), float(atol) / rhs_norm)
    prev_u = prev_r = None
    updates = mv = rmv = 0
    hist, counts = [], []
    budget = None if max_operator_actions is None else int(max_operator_actions)
    while True:
        r = matvec(u) - rhs
        mv += 1
        rel = float(np.linalg.norm(r)) / rhs_norm
        hist.append(rel)
        counts.append(mv + rmv)
        if not np.isfinite(rel):
            status = "nonfinite"
            break
        if rel < tol:
            status = "converged"
            break
        if divergence_guard is not None and rel > float(divergence_guard):
            status = "divergence_guard"
            break
        if budget is not None and mv + rmv >= budget:
            status = "max_operator_actions"
            break
        if updates >= int(max_iter):
            status = "max_iter"
            break
        if budget is not None and mv + rmv + 2 > budget:
            status = "max_operator_actions"
            break
        g = rmatvec(r)
        rmv += 1
        Hg = matvec(g)
        mv += 1
        a11 = rdot(Hg, Hg)
        if not np.isfinite(a11) or a11 <= 0.0:
            status = "breakdown_gradient"
            break
        if prev_u is None:
            h = rdot(g, g) / a11
            nxt = u - cdt(h) * g
        else:
            dr = r - prev_r
            a00 = rdot(dr, dr)
            a01 = rdot(dr, Hg)
            b0 = rdot(r, dr)
            b1 = rdot(r, Hg)
            det = a00 * a11 - a01 * a01
            scale = max(abs(a00 * a11), abs(a01 * a01), 1.0)
            if abs(det) <= 1e-14 * scale:
                t, h = 0.0, b1 / a11
            else:
                t = (b0 * a11 - b1 * a01) / det
                h = (a00 * b1 - a01 * b0) / det
            nxt = u - cdt(t) * (u - prev_u) - cdt(h) * g
        prev_u, prev_r = u, r
        u = nxt
        updates += 1
    return _result(u, updates, hist, status, mv, rmv, counts)


def true_relative_residual(matvec, u, rhs) -> float:
    """``||A u - f|| / ||f||`` (reference ``src/em3d/experiments/stationary_validation.py:172-180``)."""
    f = float(np.linalg.norm(rhs))
    res = float(np.linalg.norm(matvec(u) - rhs))
    return res if f == 0.0 else res / f
