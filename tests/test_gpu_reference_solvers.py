"""The drop-in boundary exercised by the reference's own code.

The reference's unmodified solvers (``em3d.BiCGStab`` / ``TwoStep`` / ``SIM``
from the copy installed in ``baseline/_ref``) drive an ``em3d_b200.Operator``
through the operator protocol they use (``operator.backend``, ``matvec``,
``rmatvec``; reference ``src/em3d/solvers/base.py:47-48``) and the
backend's array namespace (``xp.zeros_like``, ``xp.vdot``, ``xp.linalg.norm``,
``xp.asarray(..).copy()``, ``be.complex_dtype(scalar) * x``, ``be.to_host``).
They must reproduce the reference's own runs on the README sphere (golden
statuses, iteration counts, histories and solutions).  The flat-vector entry
points (``matvec_flat``, ``rmatvec_flat``, ``iteration_matvec_flat``;
reference ``src/em3d/operator.py:400-409``, ``src/em3d/layout.py:14-39``) are
checked against the oracle.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import ROOT, golden, rel_err

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "baseline", "_ref")


def _reference():
    if not os.path.isdir(os.path.join(REF, "em3d")):
        pytest.skip("the reference is not installed in baseline/_ref")
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import em3d

    return em3d


def _sphere16(prec):
    import em3d_b200 as e

    g = golden("em_sphere16.npz")
    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    prob = e.Problem(grid=grid, eps_tensor=g[f"chi_{prec}"], wave=g[f"wave_{prec}"], k0=4.0, volume=1.0)
    return be, prob, e.Operator(prob)


@pytest.mark.parametrize("prec", ["double", "single"])
@pytest.mark.parametrize("solver", ["bicgstab", "twostep", "sim"])
def test_reference_solvers_run_unmodified_on_b200_operator(solver, prec):
    em3d = _reference()
    be, prob, op = _sphere16(prec)
    sol = golden("solvers.json")
    ref = sol[f"sphere16_{solver}_{prec}"]
    rtol = 1e-8 if prec == "double" else 1e-5
    if solver == "bicgstab":
        s = em3d.BiCGStab(em3d.SolverConfig(max_iter=200, rtol=rtol))
    elif solver == "twostep":
        s = em3d.TwoStep(em3d.SolverConfig(max_iter=200, rtol=rtol))
    else:
        g0 = sol[f"sphere16_gamma0_{prec}"]
        s = em3d.SIM(em3d.SolverConfig(max_iter=200, rtol=rtol, mu=complex(*g0["mu"]), radius=g0["radius"]))
    res = s.solve(op, prob.wave)
    assert res.status == ref["status"]
    assert res.iterations == ref["iterations"]
    assert res.matvec_count == ref["matvec_count"]
    assert res.rmatvec_count == ref["rmatvec_count"]
    htol = 1e-7 if prec == "double" else 2e-3
    np.testing.assert_allclose(res.residual_history, ref["residual_history"], rtol=htol)
    u = be.to_host(res.u)
    assert u.dtype == be.complex_dtype
    assert rel_err(u, golden(f"sol_sphere16_{solver}_{prec}_u.npy")) < (1e-9 if prec == "double" else 1e-4)


@pytest.mark.parametrize("prec,tol", [("double", 1e-12), ("single", 1e-5)])
def test_flat_vector_entry_points_against_oracle(prec, tol):
    from oracle import em as oem

    g = golden("em_aniso12.npz")
    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    import em3d_b200 as e

    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
    chi = g["chi_double"]
    cdt = be.complex_dtype
    prob = e.Problem(grid=grid, eps_tensor=chi.astype(cdt), wave=g["wave_double"].astype(cdt), k0=k, volume=1.0)
    op = e.Operator(prob)
    u = g["u_double"]
    kh = oem.kernel_hat(N, L, k)
    flat = oem.flatten_field(u).astype(cdt)
    assert rel_err(be.to_host(op.matvec_flat(flat)), oem.flatten_field(oem.matvec(chi, u, kh, N))) < tol
    assert rel_err(be.to_host(op.rmatvec_flat(flat)),
                   oem.flatten_field(oem.rmatvec(chi, u, N, khat=kh))) < tol
    mu = 1.3 - 0.2j
    want = oem.flatten_field(u) - oem.flatten_field(oem.matvec(chi, u, kh, N)) / mu
    assert rel_err(be.to_host(op.iteration_matvec_flat(flat, mu=mu)), want) < tol
    with pytest.raises(ValueError, match="mu must be non-zero"):
        op.iteration_matvec_flat(flat, mu=0.0)
