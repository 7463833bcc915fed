"""Problems of uneven grid sizes in one application (``em3d_b200.groups.UnevenGroup``).

Every pass is one launch over all sizes; each entry must equal its own
problem's operator (which the operator tests pin to the reference and the
oracle), the padding of each row must stay untouched, stopped entries must be
skipped, and batched solves over the group must reach each problem's own
solution.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

SPHERES = [((0.0, 0.0, 0.0), 0.25, 2.0 + 0.05j, 4.0), ((0.05, -0.05, 0.0), 0.2, 3.0 + 0.0j, 6.5),
           ((-0.05, 0.0, 0.05), 0.3, 1.6 + 0.1j, 3.0), ((0.02, 0.03, -0.04), 0.22, 2.4 + 0.02j, 5.0)]


def _problems(sizes, prec="double", acoustic=False, rotated=()):
    """One problem per grid size (cycling through SPHERES); entries listed in
    ``rotated`` get a rotated anisotropic (symmetric) contrast."""
    import em3d_b200 as e
    from em3d_b200 import scenes
    from em3d_b200.acoustics import AcousticProblem

    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    out = []
    for i, N in enumerate(sizes):
        c, r, eps, k0 = SPHERES[i % len(SPHERES)]
        grid = e.Grid(N=N, L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
        wave = scenes.plane_wave(grid, k=k0, orient=(0.0, 0.6, 0.8), amplitude=(1.0, 0.0, 0.0))
        if acoustic:
            eta = scenes.sample_scene_eta(grid, [scenes.EllipsoidShape(c, (r,) * 3, None, eps)])
            out.append(AcousticProblem(grid=grid, eta=eta, wave=wave[0].contiguous(), k0=k0, volume=1.0))
            continue
        if i in rotated:
            rot = np.linalg.qr(np.random.default_rng(i).standard_normal((3, 3)))[0]
            eps_t = rot @ np.diag([eps, 1.5 * eps, 0.8 * eps]) @ rot.T
            eps_t = 0.5 * (eps_t + eps_t.T)  # exactly symmetric
            shape = scenes.EllipsoidShape(c, (r, 0.8 * r, 0.9 * r), rot, eps_t)
        else:
            shape = scenes.EllipsoidShape(c, (r,) * 3, None, eps)
        out.append(e.Problem(grid=grid, eps_tensor=scenes.sample_scene(grid, [shape]), wave=wave, k0=k0,
                             volume=1.0))
    return out


def _check_entries(group, probs, x, tol, acoustic=False):
    import em3d_b200 as e
    from em3d_b200.acoustics import AcousticOperator

    y, ya = group.matvec(x), group.rmatvec(x)
    for b in range(len(group)):
        p = probs[group.order[b]]
        assert group.problems[b] is p
        op = AcousticOperator(p) if acoustic else e.Operator(p)
        xb = group.entry_field(x, b)
        assert rel_err(group.entry_field(y, b).cpu().numpy(), op.matvec(xb).cpu().numpy()) < tol, b
        assert rel_err(group.entry_field(ya, b).cpu().numpy(), op.rmatvec(xb).cpu().numpy()) < tol, b
        m = group.entry_lengths[b]
        if m < group.n:
            # the padding beyond the problem's field is left as it was (zero)
            assert y[b, m:].abs().max().item() == 0.0, b
    return y


@pytest.mark.parametrize("prec,sizes,tol", [
    ("double", [(32, 32, 32), (16, 16, 16), (16, 32, 48), (80, 80, 80), (32, 32, 32), (48, 48, 48)], 1e-13),
    ("single", [(48, 48, 48), (32, 32, 32), (32, 48, 64), (80, 80, 80), (32, 32, 32)], 2e-6),
])
def test_uneven_em_equals_single_operators(prec, sizes, tol):
    import torch

    from em3d_b200.groups import UnevenGroup

    probs = _problems(sizes, prec)
    group = UnevenGroup(probs)
    assert [tuple(p.grid.N) for p in group.problems] == sorted(tuple(N) for N in sizes)
    assert group.chi_layout == "isotropic"
    x = group.pack([torch.randn(group.problem_shape(b), dtype=group._tc, device="cuda") for b in range(len(group))])
    _check_entries(group, probs, x, tol)


@pytest.mark.parametrize("rotated,layout", [((1,), "symmetric"), ((0, 1, 2), "symmetric")])
def test_uneven_em_contrast_layouts(rotated, layout):
    """A group stores every contrast in the smallest layout that fits all of
    them (isotropic spheres join a rotated anisotropic one as symmetric)."""
    import torch

    from em3d_b200.groups import UnevenGroup

    probs = _problems([(16, 16, 16), (32, 16, 48), (32, 32, 32)], "double", rotated=rotated)
    group = UnevenGroup(probs)
    assert group.chi_layout == layout
    x = group.pack([torch.randn(group.problem_shape(b), dtype=group._tc, device="cuda") for b in range(len(group))])
    _check_entries(group, probs, x, 1e-13)


def test_uneven_em_full_contrast():
    """A non-symmetric contrast makes the group store full tensors."""
    import torch

    import dataclasses

    from em3d_b200.groups import UnevenGroup

    probs = _problems([(16, 16, 16), (32, 32, 32)], "double")
    chi = probs[1].eps_tensor.clone()
    chi[0, 1] += 0.1 * (chi[0, 0] != 0)
    probs[1] = dataclasses.replace(probs[1], eps_tensor=chi)
    group = UnevenGroup(probs)
    assert group.chi_layout == "full"
    x = group.pack([torch.randn(group.problem_shape(b), dtype=group._tc, device="cuda") for b in range(len(group))])
    _check_entries(group, probs, x, 1e-13)


@pytest.mark.parametrize("prec,sizes,tol", [
    ("double", [(16, 16, 16), (32, 16, 48), (64, 32, 32)], 1e-13),
    ("single", [(32, 32, 32), (64, 48, 32), (96, 64, 80)], 2e-6),
])
def test_uneven_acoustic_equals_single_operators(prec, sizes, tol):
    import torch

    from em3d_b200.groups import UnevenGroup

    probs = _problems(sizes, prec, acoustic=True)
    group = UnevenGroup(probs, acoustic=True)
    x = group.pack([torch.randn(group.problem_shape(b), dtype=group._tc, device="cuda") for b in range(len(group))])
    _check_entries(group, probs, x, tol, acoustic=True)


def test_uneven_entry_against_oracle():
    """One entry of a mixed-size application against the oracle directly."""
    import torch

    from em3d_b200.groups import UnevenGroup
    from oracle import em as oem

    probs = _problems([(32, 32, 32), (16, 32, 48)], "double")
    group = UnevenGroup(probs)
    b = [tuple(p.grid.N) for p in group.problems].index((16, 32, 48))
    rng = np.random.default_rng(3)
    xs = [rng.standard_normal(group.problem_shape(i)) + 1j * rng.standard_normal(group.problem_shape(i))
          for i in range(len(group))]
    x = group.pack([torch.as_tensor(v) for v in xs])
    y = group.matvec(x)
    p = group.problems[b]
    kh = oem.kernel_hat((16, 32, 48), (1.0, 1.0, 1.0), p.k0)
    ref = oem.matvec(p.eps_tensor.cpu().numpy(), xs[b], kh, (16, 32, 48))
    assert rel_err(group.entry_field(y, b).cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize("prec", ["double", "single"])
def test_uneven_stopped_entries_are_left_untouched(prec):
    import torch

    from em3d_b200.groups import UnevenGroup

    sizes = [(32, 32, 32), (48, 48, 48), (32, 32, 32), (64, 32, 48)]
    group = UnevenGroup(_problems(sizes, prec))
    x = group.pack([torch.randn(group.problem_shape(b), dtype=group._tc, device="cuda") for b in range(len(group))])
    full = group.matvec(x)
    flags = torch.tensor([0, 1, 0, 1], dtype=torch.int32, device="cuda")
    out = torch.full_like(x, 7.0 + 3.0j)
    group.apply_into(x, out, entry_done=(flags.data_ptr(), 4))
    torch.cuda.synchronize()
    for b in range(len(group)):
        if flags[b]:
            assert torch.equal(out[b], torch.full_like(x[b], 7.0 + 3.0j)), b
        else:
            m = group.entry_lengths[b]
            assert torch.equal(out[b, :m], full[b, :m]), b


def test_uneven_bicgstab_matches_problem_by_problem():
    """Each entry's batched run is its single run: same status, iterations,
    residual history and solution (the (32, 16, 48) problem stagnates near
    1e-3 in both, the others converge; the stagnating entry keeps running
    while the others have stopped and skip their work)."""
    import em3d_b200 as e
    from em3d_b200.groups import UnevenGroup
    from em3d_b200.solvers import BiCGStab, SolverConfig

    probs = _problems([(16, 16, 16), (32, 16, 48), (16, 16, 16), (32, 32, 32)], "double")
    group = UnevenGroup(probs)
    s = BiCGStab(SolverConfig(max_iter=300, rtol=1e-9))
    s.fuse_dots = False  # the batched kernels' inner products, for a like-for-like single solve
    batch = s.solve_batch(group, group.waves())
    iters = []
    for b in range(len(group)):
        p = group.problems[b]
        single = s.solve(e.Operator(p), p.wave)
        assert batch[b].status == single.status, b
        assert batch[b].iterations == single.iterations, b
        np.testing.assert_allclose(batch[b].residual_history, single.residual_history, rtol=1e-9)
        assert batch[b].u.shape == p.wave.shape
        assert rel_err(batch[b].u.cpu().numpy(), single.u.cpu().numpy()) < 1e-8, b
        iters.append(single.iterations)
    done = [b for b in range(len(group)) if batch[b].status == "converged"]
    assert len(done) == 3
    res = group.true_relative_residuals(group.pack([r.u for r in batch]), group.waves())
    assert max(res[b] for b in done) < 1e-9
    assert len(set(iters)) > 1


def test_uneven_mixed_solve_reaches_each_problem_solution():
    """FP32 iterations with FP64 reliable updates over an uneven group (its
    twin converted on the device) reach every problem's FP64 solution."""
    import em3d_b200 as e
    from em3d_b200.groups import UnevenGroup
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    probs = _problems([(32, 32, 32), (48, 48, 48), (32, 32, 32), (64, 64, 64), (48, 48, 48)], "double")
    group = UnevenGroup(probs)
    low = group.with_precision(e.Precision.SINGLE)
    cfg = SolverConfig(max_iter=300, rtol=1e-8)
    res = MixedBiCGStab(cfg).solve_batch(group, group.waves(), operator_low=low)
    for b in range(len(group)):
        p = group.problems[b]
        one = MixedBiCGStab(cfg).solve(e.Operator(p), p.wave)
        assert res[b].status == one.status == "converged", b
        assert abs(res[b].iterations - one.iterations) <= 2, b
        assert rel_err(res[b].u.cpu().numpy(), one.u.cpu().numpy()) < 1e-6, b
    assert group.true_relative_residuals(group.pack([r.u for r in res]), group.waves()).max() < 1e-8


def test_grouped_solver_single_launch_in_input_order():
    import em3d_b200 as e
    from em3d_b200.groups import GroupedSolver
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig

    probs = _problems([(32, 32, 32), (48, 48, 48), (32, 16, 48), (48, 48, 48), (32, 32, 32)], "double")
    cfg = SolverConfig(max_iter=300, rtol=1e-8)
    one = GroupedSolver(probs, lambda: MixedBiCGStab(cfg), low_precision=e.Precision.SINGLE, single_launch=True)
    per = GroupedSolver(probs, lambda: MixedBiCGStab(cfg), low_precision=e.Precision.SINGLE)
    a, b = one.solve(), per.solve()
    for i, p in enumerate(probs):
        assert a[i].u.shape == p.wave.shape, i
        assert a[i].status == b[i].status == "converged", i
        assert rel_err(a[i].u.cpu().numpy(), b[i].u.cpu().numpy()) < 1e-6, i


def test_uneven_group_on_benchmark_sizes():
    """The 48-problem workload's sizes (32..80 cells per axis), a sample of
    eight problems: every entry equals its own operator."""
    import torch

    from em3d_b200 import workloads
    from em3d_b200.groups import UnevenGroup

    probs = workloads.uneven_sphere_problems("single", 8, seed=0)
    group = UnevenGroup(probs)
    assert len({tuple(p.grid.N) for p in probs}) >= 3
    x = group.pack([torch.randn(group.problem_shape(b), dtype=group._tc, device="cuda") for b in range(len(group))])
    _check_entries(group, probs, x, 2e-6)


def test_uneven_group_rejects_unsupported():
    from em3d_b200.groups import UnevenGroup

    with pytest.raises(ValueError, match="uneven"):
        UnevenGroup(_problems([(16, 16, 16), (40, 40, 40)], "double"))
    with pytest.raises(ValueError, match="at most 8"):
        UnevenGroup(_problems([(16, 16, n) for n in (16, 32, 48, 64, 80, 96, 128)] + [(32, 16, 16), (48, 16, 16)],
                              "double"))


@pytest.mark.parametrize("variant", [-1, 0, 6])
def test_uneven_x_pass_choices_agree(variant):
    """The complex64 EM application runs its x pass pipelined (persistent
    CTAs, field slab by TMA) by default and one tile per CTA when a
    non-pipelined x-pass variant is selected; both equal the single
    operators."""
    import torch

    from em3d_b200 import tune
    from em3d_b200.groups import UnevenGroup

    probs = _problems([(64, 64, 64), (32, 32, 32), (80, 80, 80), (48, 48, 48), (32, 32, 32)], "single")
    group = UnevenGroup(probs)
    x = group.pack([torch.randn(group.problem_shape(b), dtype=group._tc, device="cuda") for b in range(len(group))])
    old = tune.get_xpass_variant()
    try:
        tune.set_xpass_variant(variant)
        y = group.matvec(x)
    finally:
        tune.set_xpass_variant(old)
    import em3d_b200 as e

    for b, p in enumerate(group.problems):
        ref = e.Operator(p).matvec(group.entry_field(x, b))
        assert rel_err(group.entry_field(y, b).cpu().numpy(), ref.cpu().numpy()) < 2e-6, b
