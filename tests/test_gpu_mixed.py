"""FP32 BiCGStab with FP64 reliable updates: converges on the FP64 true
residual to the FP64 solution, without the restart penalty of defect
correction."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu


def _unfused(solver):
    """A single-right-hand-side solver that forms its inner products with the
    separate kernels, as the batched solves do, so that the two follow the
    same arithmetic (the fused path is compared with them in
    test_gpu_solvers.py)."""
    solver.fuse_dots = False
    return solver


def _sphere16():
    import em3d_b200 as e

    g = golden("em_sphere16.npz")
    be = e.Backend.b200(e.Precision.DOUBLE)
    grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    prob = e.Problem(grid=grid, eps_tensor=g["chi_double"], wave=g["wave_double"], k0=4.0, volume=1.0)
    return be, prob, e.Operator(prob)


def _aniso32():
    import em3d_b200 as e
    from em3d_b200 import workloads

    case = workloads.aniso_ellipsoid_em(32, "double", k0=12.0)
    be = e.Backend.b200(e.Precision.DOUBLE)
    grid = e.Grid(N=case.N, L=case.L, center=case.center, backend=be)
    prob = e.Problem(grid=grid, eps_tensor=case.chi, wave=case.wave, k0=case.k0, volume=1.0)
    return be, prob, e.Operator(prob)


@pytest.mark.parametrize("make", [_sphere16, _aniso32])
def test_mixed_reaches_fp64_solution(make):
    from em3d_b200.solvers import BiCGStab, DefectCorrection, MixedBiCGStab, SolverConfig, true_relative_residual

    be, prob, op = make()
    ref = BiCGStab(SolverConfig(max_iter=500, rtol=1e-12)).solve(op, prob.wave)
    fp64 = BiCGStab(SolverConfig(max_iter=500, rtol=1e-9)).solve(op, prob.wave)
    dc = DefectCorrection(SolverConfig(max_iter=500, rtol=1e-9)).solve(op, prob.wave)
    mx = MixedBiCGStab(SolverConfig(max_iter=500, rtol=1e-9))
    res = mx.solve(op, prob.wave)
    assert res.converged and res.status == "converged"
    assert true_relative_residual(op, res.u, prob.wave) < 1e-9
    assert res.residual_history[-1] < 1e-9 and res.residual_history[0] == pytest.approx(1.0)
    assert rel_err(be.to_host(res.u), be.to_host(ref.u)) < 1e-7
    # FP32 arithmetic costs some iterations against FP64 BiCGStab, but no more
    # than restarting does in defect correction
    assert res.iterations <= 1.3 * fp64.iterations + 2
    assert res.iterations <= sum(dc.inner_iterations) + 1
    # from the zero guess the first residual is f itself: one FP64 application per update
    assert res.fp64_matvecs == res.outer_iterations
    assert res.matvec_count == res.fp64_matvecs + res.fp32_matvecs
    # a repeated solve (cached buffers and graph) gives the same answer
    again = mx.solve(op, prob.wave)
    assert again.residual_history == res.residual_history and again.iterations == res.iterations


def test_mixed_warm_start_and_fallback():
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    be, prob, op = _sphere16()
    mx = MixedBiCGStab(SolverConfig(max_iter=300, rtol=1e-10))
    cold = mx.solve(op, prob.wave)
    warm = mx.solve(op, prob.wave, x0=cold.u * (1 + 1e-6))
    assert warm.converged and not warm.guess_rejected and warm.residual_history[0] < 1e-4
    assert warm.iterations < cold.iterations
    bad = mx.solve(op, prob.wave, x0=prob.wave * 40.0)
    assert bad.guess_rejected and bad.converged and bad.residual_history[0] == 1.0
    assert rel_err(be.to_host(bad.u), be.to_host(cold.u)) < 1e-8


def test_mixed_zero_rhs_and_batch_rejected():
    import torch

    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    be, prob, op = _sphere16()
    mx = MixedBiCGStab(SolverConfig(max_iter=50, rtol=1e-8))
    z = mx.solve(op, torch.zeros_like(prob.wave))
    assert z.converged and z.iterations == 0 and float(z.u.abs().max()) == 0.0
    with pytest.raises(NotImplementedError):
        mx.solve(op, torch.stack([prob.wave, prob.wave]))
    with pytest.raises(ValueError):
        MixedBiCGStab(SolverConfig(), delta=1.5)


def test_mixed_budget_stops_with_max_iter():
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    be, prob, op = _aniso32()
    res = MixedBiCGStab(SolverConfig(max_iter=3, rtol=1e-12)).solve(op, prob.wave)
    assert not res.converged and res.status == "max_iter" and res.iterations <= 3
    assert np.isfinite(res.residual_history[-1])


def _same_as_single(batch, singles):
    for b, (got, one) in enumerate(zip(batch, singles)):
        assert got.status == one.status, b
        assert got.iterations == one.iterations and got.inner_iterations == one.inner_iterations, b
        assert got.fp64_matvecs == one.fp64_matvecs and got.fp32_matvecs == one.fp32_matvecs, b
        assert got.residual_action_counts == one.residual_action_counts, b
        np.testing.assert_allclose(got.residual_history, one.residual_history, rtol=1e-6, atol=1e-14)
        assert rel_err(got.u.cpu().numpy(), one.u.cpu().numpy()) < 1e-6, b


def test_mixed_batch_matches_single_solves():
    """Many right-hand sides on one operator: every entry runs the cycles of
    its single solve (a zero right-hand side comes back converged at u = 0)."""
    import torch

    from em3d_b200 import workloads
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    be, prob, op = _aniso32()
    waves = workloads.plane_wave_batch(prob.grid.host_axes, 12.0, 2, dtype=np.complex128)
    rhs = torch.cat([torch.as_tensor(waves, device="cuda"), torch.zeros_like(prob.wave)[None]])
    mx = MixedBiCGStab(SolverConfig(max_iter=500, rtol=1e-9))
    batch = mx.solve_batch(op, rhs)
    assert len(batch) == rhs.shape[0] == 5   # two directions x two polarisations + the zero one
    singles = [_unfused(MixedBiCGStab(SolverConfig(max_iter=500, rtol=1e-9))).solve(op, rhs[b]) for b in range(5)]
    _same_as_single(batch, singles)
    assert batch[4].converged and batch[4].iterations == 0 and float(batch[4].u.abs().max()) == 0.0
    # a second batch through the cached engines gives the same answers
    again = mx.solve_batch(op, rhs)
    _same_as_single(again, singles)


def test_mixed_group_matches_problem_by_problem():
    """A group of problems (each its own contrast and wave number) solved at
    once, entries that finish early skipped: each entry as its own solve."""
    import em3d_b200 as e
    from em3d_b200 import workloads
    from em3d_b200.groups import OperatorGroup
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    probs = [p for p in workloads.uneven_sphere_problems("double", 12, seed=5, sizes=(24,))]
    group = OperatorGroup(probs)
    cfg = SolverConfig(max_iter=500, rtol=1e-8)
    batch = MixedBiCGStab(cfg).solve_batch(group, group.waves())
    singles = [_unfused(MixedBiCGStab(cfg)).solve(e.Operator(p), p.wave) for p in probs]
    _same_as_single(batch, singles)
    assert all(r.converged for r in batch)
    assert len({r.iterations for r in batch}) > 1
