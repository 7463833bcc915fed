"""Batched solves: many right-hand sides sharing one operator (one spectrum).

Each right-hand side of a batch keeps its own Krylov scalars and stops on its
own, so it must reproduce the single right-hand-side solve: same status,
iteration count and action counts, and the same history and solution up to
the rounding differences of the batched reductions (none here: the same
kernels reduce each right-hand side in the same order).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu


def _setup_batch(prec="double", n_dirs=3):
    import torch

    import em3d_b200 as e
    from em3d_b200 import workloads

    g = golden("em_sphere16.npz")
    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    prob = e.Problem(grid=grid, eps_tensor=g[f"chi_{prec}"], wave=g[f"wave_{prec}"], k0=4.0, volume=1.0)
    op = e.Operator(prob)
    waves = workloads.plane_wave_batch(grid.host_axes, 4.0, n_dirs, dtype=be.complex_dtype)
    rhs = torch.as_tensor(waves, device="cuda")
    return be, op, rhs


@pytest.mark.parametrize("solver", ["bicgstab", "twostep", "sim"])
def test_batched_solver_matches_single_rhs_solves(solver):
    import torch

    from em3d_b200.solvers import SIM, BiCGStab, SolverConfig, TwoStep

    be, op, rhs = _setup_batch()
    # add a zero right-hand side: it must come back converged with u = 0
    rhs = torch.cat([rhs, torch.zeros_like(rhs[:1])])
    if solver == "bicgstab":
        s = BiCGStab(SolverConfig(max_iter=200, rtol=1e-9))
        s.fuse_dots = False  # the batched kernels' inner products, for a like-for-like single solve
    elif solver == "twostep":
        s = TwoStep(SolverConfig(max_iter=200, rtol=1e-8))
    else:
        g0 = golden("solvers.json")["sphere16_gamma0_double"]
        s = SIM(SolverConfig(max_iter=200, rtol=1e-8, mu=complex(*g0["mu"]), radius=g0["radius"]))
    batch = s.solve_batch(op, rhs)
    assert len(batch) == rhs.shape[0]
    for b in range(rhs.shape[0]):
        single = s.solve(op, rhs[b])
        got = batch[b]
        assert got.status == single.status, b
        assert got.iterations == single.iterations, b
        assert got.matvec_count == single.matvec_count and got.rmatvec_count == single.rmatvec_count
        assert got.residual_action_counts == single.residual_action_counts
        np.testing.assert_allclose(got.residual_history, single.residual_history, rtol=1e-9)
        if float(torch.linalg.vector_norm(single.u)) > 0:  # agreement at the solve tolerance
            assert rel_err(be.to_host(got.u), be.to_host(single.u)) < 1e-8
    assert batch[-1].status == "converged" and float(torch.linalg.vector_norm(batch[-1].u)) == 0.0


def test_batched_defect_correction_matches_single():
    import em3d_b200 as e
    from em3d_b200.solvers import DefectCorrection, SolverConfig, true_relative_residual

    be, op, rhs = _setup_batch(n_dirs=2)
    op32 = op.with_precision(e.Precision.SINGLE)
    dc = DefectCorrection(SolverConfig(max_iter=300, rtol=1e-9))
    batch = dc.solve_batch(op, rhs, operator_low=op32)
    for b in range(rhs.shape[0]):
        single = dc.solve(op, rhs[b], operator_low=op32)
        assert batch[b].converged and single.converged
        assert true_relative_residual(op, batch[b].u, rhs[b]) < 1e-9
        assert rel_err(be.to_host(batch[b].u), be.to_host(single.u)) < 1e-8


def test_defect_correction_reaches_fp64_accuracy_against_oracle():
    """Mixed precision result against a complex128 reference solve (the oracle)."""
    import em3d_b200 as e
    from em3d_b200.solvers import DefectCorrection, SolverConfig
    from oracle import em as oem
    from oracle import solvers as osol

    g = golden("em_aniso12.npz")
    be = e.Backend.b200(e.Precision.DOUBLE)
    grid = e.Grid(N=(12, 12, 12), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    prob = e.Problem(grid=grid, eps_tensor=g["chi_double"], wave=g["wave_double"], k0=12.0, volume=1.0)
    op = e.Operator(prob)
    res = DefectCorrection(SolverConfig(max_iter=500, rtol=1e-10)).solve(op, prob.wave)
    assert res.converged and res.outer_iterations >= 1
    kh = oem.kernel_hat((12, 12, 12), (1.0, 1.0, 1.0), 12.0)
    ref = osol.bicgstab(lambda x: oem.matvec(g["chi_double"], x, kh, (12, 12, 12)), g["wave_double"],
                        max_iter=500, rtol=1e-12)
    assert rel_err(be.to_host(res.u), ref["u"]) < 1e-8


def test_batched_acoustic_bicgstab():
    import torch

    import em3d_b200 as e
    from em3d_b200 import acoustics as ea
    from em3d_b200.solvers import BiCGStab, SolverConfig

    g = golden("ac_spheres16.npz")
    be = e.Backend.b200(e.Precision.DOUBLE)
    grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    prob = ea.make_acoustic_problem(grid, g["eta_double"], k0=20.0)
    op = ea.AcousticOperator(prob)
    dirs = [(0, 0, 1), (1, 0, 0), (0.6, 0.8, 0.0)]
    rhs = torch.stack([ea.plane_wave_scalar(grid, k=20.0, direction=d) for d in dirs])
    s = BiCGStab(SolverConfig(max_iter=300, rtol=1e-8))
    s.fuse_dots = False  # the batched kernels' inner products, for a like-for-like single solve
    batch = s.solve_batch(op, rhs)
    for b in range(len(dirs)):
        single = s.solve(op, rhs[b])
        assert batch[b].status == single.status and batch[b].iterations == single.iterations
        assert rel_err(be.to_host(batch[b].u), be.to_host(single.u)) < 1e-9
