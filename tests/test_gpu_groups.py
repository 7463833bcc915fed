"""Groups of problems on one grid (``em3d_b200.groups``).

Entry b of a group is problem b with its own contrast and spectrum; applying
the group must give each problem's own operator, batched solves over a group
must reproduce the problem-by-problem solves, and entries flagged as stopped
must be left untouched.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

SPHERES = [((0.0, 0.0, 0.0), 0.25, 2.0 + 0.05j, 4.0), ((0.05, -0.05, 0.0), 0.2, 3.0 + 0.0j, 6.5),
           ((-0.05, 0.0, 0.05), 0.3, 1.6 + 0.1j, 3.0)]


def _unfused(solver):
    """A single-right-hand-side solver that forms its inner products with the
    separate kernels, as the batched solves do (same arithmetic)."""
    solver.fuse_dots = False
    return solver


def _problems(N, prec="double", acoustic=False):
    import em3d_b200 as e
    from em3d_b200 import scenes
    from em3d_b200.acoustics import AcousticProblem

    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    grid = e.Grid(N=N, L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    out = []
    for c, r, eps, k0 in SPHERES:
        shape = scenes.EllipsoidShape(c, (r,) * 3, None, eps)
        wave = scenes.plane_wave(grid, k=k0, orient=(0.0, 0.6, 0.8), amplitude=(1.0, 0.0, 0.0))
        if acoustic:
            eta = scenes.sample_scene_eta(grid, [shape])
            out.append(AcousticProblem(grid=grid, eta=eta, wave=wave[0].contiguous(), k0=k0, volume=1.0))
        else:
            out.append(e.Problem(grid=grid, eps_tensor=scenes.sample_scene(grid, [shape]), wave=wave, k0=k0,
                                 volume=1.0))
    return out


@pytest.mark.parametrize("N", [(16, 16, 16), (12, 10, 14)])
@pytest.mark.parametrize("prec,tol", [("double", 1e-13), ("single", 1e-6)])
def test_em_group_equals_single_operators(N, prec, tol):
    import torch

    import em3d_b200 as e
    from em3d_b200.groups import OperatorGroup

    probs = _problems(N, prec)
    group = OperatorGroup(probs)
    x = torch.randn((len(probs), 3) + N, dtype=group._tc, device="cuda")
    y, ya = group.matvec(x), group.rmatvec(x)
    for b, p in enumerate(probs):
        op = e.Operator(p)
        assert rel_err(y[b].cpu().numpy(), op.matvec(x[b]).cpu().numpy()) < tol, b
        assert rel_err(ya[b].cpu().numpy(), op.rmatvec(x[b]).cpu().numpy()) < tol, b


@pytest.mark.parametrize("prec,tol", [("double", 1e-13), ("single", 1e-6)])
def test_acoustic_group_equals_single_operators(prec, tol):
    import torch

    from em3d_b200.acoustics import AcousticOperator
    from em3d_b200.groups import AcousticOperatorGroup

    N = (16, 12, 10)
    probs = _problems(N, prec, acoustic=True)
    group = AcousticOperatorGroup(probs)
    x = torch.randn((len(probs),) + N, dtype=group._tc, device="cuda")
    y, ya = group.matvec(x), group.rmatvec(x)
    for b, p in enumerate(probs):
        op = AcousticOperator(p)
        assert rel_err(y[b].cpu().numpy(), op.matvec(x[b]).cpu().numpy()) < tol, b
        assert rel_err(ya[b].cpu().numpy(), op.rmatvec(x[b]).cpu().numpy()) < tol, b


def test_group_rejects_mixed_grids():
    from em3d_b200.groups import OperatorGroup, group_by_grid

    a, b = _problems((16, 16, 16)), _problems((12, 10, 14))
    with pytest.raises(ValueError, match="same grid"):
        OperatorGroup([a[0], b[0]])
    groups = group_by_grid([a[0], b[0], a[1], b[1], a[2]])
    assert [idx for idx, _ in groups.values()] == [[0, 2, 4], [1, 3]]
    assert [len(g) for _, g in groups.values()] == [3, 2]


def test_grouped_bicgstab_matches_problem_by_problem():
    import em3d_b200 as e
    from em3d_b200.groups import OperatorGroup
    from em3d_b200.solvers import BiCGStab, SolverConfig

    probs = _problems((16, 16, 16))
    group = OperatorGroup(probs)
    s = BiCGStab(SolverConfig(max_iter=300, rtol=1e-9))
    s.fuse_dots = False  # the batched kernels' inner products, for a like-for-like single solve
    batch = s.solve_batch(group, group.waves())
    iters = []
    for b, p in enumerate(probs):
        single = s.solve(e.Operator(p), p.wave)
        assert batch[b].status == single.status == "converged", b
        assert batch[b].iterations == single.iterations, b
        assert batch[b].matvec_count == single.matvec_count, b
        np.testing.assert_allclose(batch[b].residual_history, single.residual_history, rtol=1e-9)
        assert rel_err(batch[b].u.cpu().numpy(), single.u.cpu().numpy()) < 1e-10
        iters.append(single.iterations)
    # the problems stop at different iterations: entry skipping is exercised
    assert len(set(iters)) > 1


def test_grouped_defect_correction_reaches_fp64_residuals():
    from em3d_b200.groups import OperatorGroup
    from em3d_b200.solvers import DefectCorrection, SolverConfig

    probs = _problems((16, 16, 16))
    group = OperatorGroup(probs)
    res = DefectCorrection(SolverConfig(max_iter=300, rtol=1e-10)).solve_batch(group, group.waves())
    assert all(r.status == "converged" for r in res)
    import torch

    u = torch.stack([r.u for r in res])
    assert group.true_relative_residuals(u, group.waves()).max() < 1e-10


@pytest.mark.parametrize("variant", [-1, 0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_stopped_entries_are_left_untouched(variant, prec):
    import torch

    from em3d_b200 import tune
    from em3d_b200.groups import OperatorGroup

    probs = _problems((16, 16, 16), prec)
    group = OperatorGroup(probs)
    x = torch.randn((len(probs), 3, 16, 16, 16), dtype=group._tc, device="cuda")
    old = tune.get_xpass_variant()
    try:
        tune.set_xpass_variant(variant)
        full = group.matvec(x)
        flags = torch.tensor([0, 1, 0], dtype=torch.int32, device="cuda")
        out = torch.full_like(x, 7.0 + 3.0j)
        group.apply_into(x, out, entry_done=(flags.data_ptr(), 4))
        torch.cuda.synchronize()
    finally:
        tune.set_xpass_variant(old)
    assert torch.equal(out[1], torch.full_like(x[1], 7.0 + 3.0j))
    assert torch.equal(out[0], full[0]) and torch.equal(out[2], full[2])


def test_acoustic_group_mixed_solve_matches_problem_by_problem():
    from em3d_b200.acoustics import AcousticOperator
    from em3d_b200.groups import AcousticOperatorGroup
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    probs = _problems((16, 12, 10), acoustic=True)
    group = AcousticOperatorGroup(probs)
    cfg = SolverConfig(max_iter=300, rtol=1e-8)
    batch = MixedBiCGStab(cfg).solve_batch(group, group.waves())
    for b, p in enumerate(probs):
        one = _unfused(MixedBiCGStab(cfg)).solve(AcousticOperator(p), p.wave)
        assert batch[b].status == one.status == "converged", b
        assert batch[b].iterations == one.iterations and batch[b].inner_iterations == one.inner_iterations, b
        assert rel_err(batch[b].u.cpu().numpy(), one.u.cpu().numpy()) < 1e-6, b


def test_grouped_solver_concurrent_equals_sequential():
    """Problems of two grid sizes: the groups' solves on their own streams at
    the same time give the sequential results, in the input order."""
    import em3d_b200 as e
    from em3d_b200.groups import GroupedSolver
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    a, b = _problems((16, 16, 16)), _problems((12, 10, 14))
    probs = [a[0], b[0], a[1], b[1], a[2], b[2]]
    cfg = SolverConfig(max_iter=300, rtol=1e-8)
    gs = GroupedSolver(probs, lambda: MixedBiCGStab(cfg), low_precision=e.Precision.SINGLE)
    seq = gs.solve(concurrent=False)
    con = gs.solve(concurrent=True)
    for i, p in enumerate(probs):
        one = _unfused(MixedBiCGStab(cfg)).solve(e.Operator(p), p.wave)
        assert seq[i].iterations == con[i].iterations == one.iterations, i
        assert rel_err(con[i].u.cpu().numpy(), seq[i].u.cpu().numpy()) == 0.0, i
        assert con[i].u.shape == p.wave.shape
