"""The per-operator autotuner of the x pass (tile width, threads per CTA,
radix plan, slab pipelining, twiddle placement, generic plan)."""
from __future__ import annotations

import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _em_op(N, prec):
    import torch
    import em3d_b200 as e

    be = e.Backend.b200(e.Precision.SINGLE if prec == "single" else e.Precision.DOUBLE)
    grid = e.Grid(N=N, L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    tc = be.precision.torch_complex
    gen = torch.Generator(device="cuda").manual_seed(7)
    chi = (torch.randn((3, 3) + N, dtype=tc, device="cuda", generator=gen) * 0.3).contiguous()
    u = torch.randn((3,) + N, dtype=tc, device="cuda", generator=gen)
    return be, e.Operator(e.Problem(grid=grid, eps_tensor=chi, wave=u, k0=6.0, volume=1.0))


def test_autotune_keeps_a_choice_per_operator():
    from em3d_b200 import tune

    be, op = _em_op((32, 32, 32), "single")
    ref = be.to_host(op.matvec(op.problem.wave))
    times = tune.autotune(op, reps=2)
    assert set(times) == set(tune.VARIANTS)
    assert op.xpass_variant in times and times[op.xpass_variant] == min(times.values())
    assert tune.get_xpass_variant() == -1  # the process-wide setting is left as it was
    assert rel_err(be.to_host(op.matvec(op.problem.wave)), ref) < 3e-6
    assert tune.get_xpass_variant() == -1
    # a second operator of another grid and precision is tuned on its own
    be2, op2 = _em_op((16, 32, 16), "double")
    ref2 = be2.to_host(op2.matvec(op2.problem.wave))
    t2 = tune.autotune(op2, reps=2)
    assert op2.xpass_variant in t2
    assert rel_err(be2.to_host(op2.matvec(op2.problem.wave)), ref2) < 1e-13
    # a third operator of the first kind reuses the cached timings
    _, op3 = _em_op((32, 32, 32), "single")
    assert tune.autotune(op3) is times and op3.xpass_variant == op.xpass_variant


def test_autotune_acoustic_and_group():
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea, tune, workloads
    from em3d_b200.groups import OperatorGroup

    be = e.Backend.b200(e.Precision.SINGLE)
    grid = e.Grid(N=(32, 32, 32), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    op = ea.AcousticOperator(ea.make_acoustic_problem(grid, workloads.acoustic_spheres_device(grid, count=5),
                                                      k0=8.0))
    times = tune.autotune(op, reps=2)
    assert 2 not in times  # the component split is EM only
    probs = workloads.uneven_sphere_problems("single", 3, seed=1, sizes=(32,))
    group = OperatorGroup(probs)
    ref = be.to_host(group.matvec(group.waves()))
    tg = tune.autotune(group, reps=2)
    assert group.xpass_variant in tg
    assert rel_err(be.to_host(group.matvec(group.waves())), ref) < 3e-6
