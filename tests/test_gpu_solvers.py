"""Device-resident solvers against the reference's own runs (golden histories)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu


def _be(prec):
    import em3d_b200 as e

    return e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)


def _sphere16(prec):
    import em3d_b200 as e

    g = golden("em_sphere16.npz")
    be = _be(prec)
    grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    prob = e.Problem(grid=grid, eps_tensor=g[f"chi_{prec}"], wave=g[f"wave_{prec}"], k0=4.0, volume=1.0)
    return be, prob, e.Operator(prob)


@pytest.mark.parametrize("prec", ["double", "single"])
@pytest.mark.parametrize("solver", ["bicgstab", "twostep", "sim"])
def test_solver_histories_match_reference(solver, prec):
    from em3d_b200.solvers import SIM, BiCGStab, SolverConfig, TwoStep, true_relative_residual

    be, prob, op = _sphere16(prec)
    sol = golden("solvers.json")
    ref = sol[f"sphere16_{solver}_{prec}"]
    rtol = 1e-8 if prec == "double" else 1e-5
    if solver == "bicgstab":
        s = BiCGStab(SolverConfig(max_iter=200, rtol=rtol))
    elif solver == "twostep":
        s = TwoStep(SolverConfig(max_iter=200, rtol=rtol))
    else:
        g0 = sol[f"sphere16_gamma0_{prec}"]
        s = SIM(SolverConfig(max_iter=200, rtol=rtol, mu=complex(*g0["mu"]), radius=g0["radius"]))
    res = s.solve(op, prob.wave)
    assert res.status == ref["status"]
    assert res.iterations == ref["iterations"]
    assert res.matvec_count == ref["matvec_count"]
    assert res.rmatvec_count == ref["rmatvec_count"]
    assert res.residual_action_counts == ref["residual_action_counts"]
    htol = 1e-7 if prec == "double" else 2e-3
    np.testing.assert_allclose(res.residual_history, ref["residual_history"], rtol=htol)
    u_ref = golden(f"sol_sphere16_{solver}_{prec}_u.npy")
    assert rel_err(be.to_host(res.u), u_ref) < (1e-9 if prec == "double" else 1e-4)
    tr = true_relative_residual(op, res.u, prob.wave)
    assert abs(tr - ref["true_relative_residual"]) < (1e-9 if prec == "double" else 1e-5)


@pytest.mark.parametrize("budget", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("solver", ["bicgstab", "twostep", "sim"])
def test_action_budgets_match_reference(solver, budget):
    import em3d_b200 as e
    from em3d_b200.solvers import SIM, BiCGStab, SolverConfig, TwoStep

    be = _be("double")
    grid = e.Grid(N=(4, 4, 4), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    chi = e.cylinder_refraction(grid, eps_real=1.1, eps_imag=0.0, radius=0.2, axis="z")
    wave = e.flat_wave_vec(grid, k=0.5, orient=(0, 0, 1), amplitude=(1, 0, 0))
    op = e.Operator(e.Problem(grid=grid, eps_tensor=chi, wave=wave, k0=0.5, volume=grid.dv * 64))
    ref = golden("solvers.json")[f"budget{budget}_{solver}"]
    if solver == "bicgstab":
        res = BiCGStab(SolverConfig(max_iter=100, max_operator_actions=budget)).solve(op, wave)
    elif solver == "twostep":
        res = TwoStep(SolverConfig(max_iter=100, max_operator_actions=budget)).solve(op, wave)
    else:
        res = SIM(SolverConfig(max_iter=100, max_operator_actions=budget, mu=2.0 + 0j, radius=1.0)).solve(op, wave)
    assert res.status == ref["status"]
    assert res.iterations == ref["iterations"]
    assert res.matvec_count == ref["matvec_count"]
    assert res.rmatvec_count == ref["rmatvec_count"]
    assert res.residual_action_counts == ref["residual_action_counts"]
    if budget == 2:  # the reference's own budget test (tests/test_solvers.py:154-176)
        assert res.operator_action_count <= budget
    np.testing.assert_allclose(res.residual_history, ref["residual_history"], rtol=1e-9)


@pytest.mark.parametrize("solver", ["bicgstab", "twostep"])
def test_acoustic_solvers_match_reference(solver):
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea
    from em3d_b200.solvers import BiCGStab, SolverConfig, TwoStep

    g = golden("ac_spheres16.npz")
    be = _be("double")
    grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    prob = ea.make_acoustic_problem(grid, g["eta_double"], k0=20.0)
    op = ea.AcousticOperator(prob)
    ref = golden("solvers.json")[f"ac16_{solver}_double"]
    cls = BiCGStab if solver == "bicgstab" else TwoStep
    res = cls(SolverConfig(max_iter=300, rtol=1e-8)).solve(op, prob.wave)
    assert res.status == ref["status"]
    assert res.iterations == ref["iterations"]
    assert res.residual_action_counts == ref["residual_action_counts"]
    if solver == "bicgstab":
        np.testing.assert_allclose(res.residual_history, ref["residual_history"], rtol=1e-6)
        assert rel_err(be.to_host(res.u), golden(f"sol_ac16_{solver}_double_u.npy")) < 1e-7
    else:
        # 300 slowly converging TwoStep updates amplify round-off chaotically: a
        # 1e-15 relative perturbation of the NumPy oracle itself departs from the
        # reference history by iteration ~16.  Compare the early history and the
        # solution at the level of the final residual (1.2e-6).
        np.testing.assert_allclose(res.residual_history[:12], ref["residual_history"][:12], rtol=1e-6)
        assert abs(res.residual_history[-1] - ref["residual_history"][-1]) < 1e-6
        assert rel_err(be.to_host(res.u), golden(f"sol_ac16_{solver}_double_u.npy")) < 2e-5


class _MatrixOperator:
    """Dense test operator on the device (the reference's mock-operator pattern,
    ``tests/test_solvers.py:14-23``)."""

    def __init__(self, A, backend):
        import torch

        self.A = torch.as_tensor(np.asarray(A, dtype=np.complex128), device="cuda")
        self.backend = backend

    def matvec(self, u):
        return self.A @ u

    def rmatvec(self, u):
        return self.A.conj().T @ u


def test_twostep_two_update_recurrence_generic_operator():
    """Reference ``tests/test_solvers.py:110-119``: a hand-written 2x2 recurrence to 1e-12."""
    from em3d_b200.solvers import SolverConfig, TwoStep

    be = _be("double")
    A = np.array([[2.0, 0.5], [1.0, 1.5]], dtype=np.complex128)
    rhs = np.array([1.0, -0.5], dtype=np.complex128)
    res = TwoStep(SolverConfig(max_iter=2, rtol=1e-15)).solve(_MatrixOperator(A, be), rhs)
    from oracle import solvers as osol

    expected = osol.twostep(lambda x: A @ x, lambda x: A.conj().T @ x, rhs, max_iter=2, rtol=1e-15)["u"]
    assert np.allclose(be.to_host(res.u), expected, rtol=1e-12, atol=1e-12)
    assert np.linalg.norm(A @ be.to_host(res.u) - rhs) < 1e-12


def test_breakdown_and_nonfinite_statuses():
    """Host-made failures: a NaN right-hand side and an operator that returns zero."""
    import torch

    from em3d_b200.solvers import BiCGStab, SolverConfig, TwoStep

    be = _be("double")
    A = np.eye(3, dtype=np.complex128)
    rhs = np.array([1.0, np.nan, 0.0], dtype=np.complex128)
    res = BiCGStab(SolverConfig(max_iter=10)).solve(_MatrixOperator(A, be), rhs)
    assert res.status == "nonfinite"
    zero = _MatrixOperator(np.zeros((3, 3), dtype=np.complex128), be)
    rhs = np.array([1.0, 2.0, 0.5], dtype=np.complex128)
    res = BiCGStab(SolverConfig(max_iter=10)).solve(zero, rhs)
    assert res.status == "breakdown_alpha"
    res = TwoStep(SolverConfig(max_iter=10)).solve(zero, rhs)
    assert res.status == "breakdown_gradient"
    del torch


def test_x0_warm_start_reaches_same_solution():
    from em3d_b200.solvers import BiCGStab, SolverConfig

    be, prob, op = _sphere16("double")
    cold = BiCGStab(SolverConfig(max_iter=200, rtol=1e-10)).solve(op, prob.wave)
    x0 = cold.u * (1 + 1e-4)
    warm = BiCGStab(SolverConfig(max_iter=200, rtol=1e-10)).solve(op, prob.wave, x0=x0)
    assert warm.converged and warm.iterations < cold.iterations
    assert rel_err(be.to_host(warm.u), be.to_host(cold.u)) < 1e-8


def test_repeated_solves_reuse_buffers_and_return_fresh_results():
    """Second and third solves reuse the captured graph and buffers; results
    of earlier solves are not overwritten and match a fresh solver."""
    import torch

    from em3d_b200 import workloads
    from em3d_b200.solvers import BiCGStab, SolverConfig

    be, prob, op = _sphere16("double")
    waves = torch.as_tensor(workloads.plane_wave_batch(prob.grid.host_axes, 4.0, 2), device="cuda")
    s = BiCGStab(SolverConfig(max_iter=200, rtol=1e-9))
    r0 = s.solve(op, waves[0])
    u0 = r0.u.clone()
    r1 = s.solve(op, waves[1])
    r2 = s.solve(op, waves[0])
    assert torch.equal(r0.u, u0)
    fresh = BiCGStab(SolverConfig(max_iter=200, rtol=1e-9)).solve(op, waves[1])
    assert r1.iterations == fresh.iterations and r1.residual_history == fresh.residual_history
    assert torch.equal(r1.u, fresh.u)
    assert r2.residual_history == r0.residual_history and torch.equal(r2.u, r0.u)


def test_solver_caches_release_old_operators():
    """Solving a stream of different problems keeps a bounded number of cached
    engines: operators of earlier problems are released."""
    import gc
    import weakref

    import em3d_b200 as e
    from em3d_b200.solvers import BiCGStab, DefectCorrection, SolverConfig

    be, prob, _ = _sphere16("double")
    bic = BiCGStab(SolverConfig(max_iter=200, rtol=1e-6))
    dc = DefectCorrection(SolverConfig(max_iter=200, rtol=1e-6))
    refs = []
    for k in (3.0, 3.5, 4.0, 4.5, 5.0):
        p = e.Problem(grid=prob.grid, eps_tensor=prob.eps_tensor, wave=prob.wave, k0=k, volume=1.0)
        op = e.Operator(p)
        assert bic.solve(op, p.wave).converged
        assert dc.solve(op, p.wave).converged
        refs.append(weakref.ref(op))
        del op, p
    gc.collect()
    assert len(bic._engines) <= bic.max_cached_engines and len(dc._cache) <= dc.max_cached
    assert all(r() is None for r in refs[:2])


def test_defect_correction_rejects_a_bad_guess():
    """A guess whose true residual exceeds ||f|| is replaced by the zero guess."""
    from em3d_b200.solvers import DefectCorrection, SolverConfig

    be, prob, op = _sphere16("double")
    dc = DefectCorrection(SolverConfig(max_iter=200, rtol=1e-8))
    cold = dc.solve(op, prob.wave)
    bad = dc.solve(op, prob.wave, x0=prob.wave * 50.0)
    assert bad.guess_rejected and bad.converged
    assert bad.residual_history[0] == 1.0
    assert rel_err(be.to_host(bad.u), be.to_host(cold.u)) < 1e-7
    good = dc.solve(op, prob.wave, x0=cold.u * (1 + 1e-5))
    assert not good.guess_rejected and good.residual_history[0] < 1e-3


@pytest.mark.parametrize("N", [(32, 32, 32), (24, 20, 40)])
def test_fused_omega_dots_match_separate_kernels(N):
    """BiCGStab and MixedBiCGStab with alpha's and omega's inner products
    formed in the operator's last pass (one right-hand side) follow the same
    iterations as with the separate alpha and omega kernels; a z axis without
    a register FFT (2 Nz = 80) falls back to the separate kernels."""
    import em3d_b200 as e
    from em3d_b200 import scenes
    from em3d_b200.solvers import BiCGStab, MixedBiCGStab, SolverConfig

    be = e.Backend.b200(e.Precision.DOUBLE)
    grid = e.Grid(N=N, L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    shape = scenes.EllipsoidShape((0.0, 0.05, 0.0), (0.3, 0.2, 0.25), None, 2.5 + 0.1j)
    wave = scenes.plane_wave(grid, k=6.0, orient=(0.0, 0.0, 1.0), amplitude=(1.0, 0.0, 0.0))
    p = e.Problem(grid=grid, eps_tensor=scenes.sample_scene(grid, [shape]), wave=wave, k0=6.0, volume=1.0)
    op = e.Operator(p)
    lo = op.with_precision(e.Precision.SINGLE)
    assert (op.dot_parts() > 0) == (N[2] != 40)
    cfg = SolverConfig(max_iter=300, rtol=1e-9)
    runs = {}
    for fuse in (True, False):
        b = BiCGStab(cfg)
        b.fuse_dots = fuse
        m = MixedBiCGStab(cfg)
        m.fuse_dots = fuse
        runs[fuse] = (b.solve(op, p.wave), m.solve(op, p.wave, operator_low=lo))
    for k in range(2):
        a, c = runs[True][k], runs[False][k]
        assert a.status == c.status == "converged"
        assert a.iterations == c.iterations and a.matvec_count == c.matvec_count
        np.testing.assert_allclose(a.residual_history, c.residual_history, rtol=1e-6)
        assert rel_err(a.u.cpu().numpy(), c.u.cpu().numpy()) < 1e-8


def test_copy_small_between_device_and_pinned_host():
    """em3d_copy_small moves a few bytes (a ragged tail included) from device
    memory to pinned host memory and back by a kernel, and refuses pageable
    host memory."""
    import torch

    from em3d_b200 import _lib

    src = torch.arange(1001, dtype=torch.int32, device="cuda").view(torch.uint8)[:4002]
    host = torch.zeros(4004, dtype=torch.uint8).pin_memory()
    stream = torch.cuda.current_stream()
    _lib.call("em3d_copy_small", host.data_ptr(), src.data_ptr(), 4002, stream.cuda_stream)
    stream.synchronize()
    assert torch.equal(host[:4002], src.cpu()) and int(host[4002:].sum()) == 0
    host[:4002] = torch.arange(4002, dtype=torch.int64).remainder(251).to(torch.uint8)
    back = torch.zeros(4004, dtype=torch.uint8, device="cuda")
    _lib.call("em3d_copy_small", back.data_ptr(), host.data_ptr(), 4002, stream.cuda_stream)
    assert torch.equal(back[:4002].cpu(), host[:4002]) and int(back[4002:].sum()) == 0
    # addresses 4-byte but not 16-byte aligned take the 4-byte word path
    host.zero_()
    _lib.call("em3d_copy_small", host.data_ptr() + 4, src.data_ptr() + 4, 998, stream.cuda_stream)
    stream.synchronize()
    assert torch.equal(host[4:1002], src[4:1002].cpu()) and int(host[:4].sum()) == 0 and int(host[1002:].sum()) == 0
    pageable = torch.zeros(16, dtype=torch.uint8)
    with pytest.raises(ValueError, match="pinned host memory"):
        _lib.call("em3d_copy_small", pageable.data_ptr(), src.data_ptr(), 16, stream.cuda_stream)


def test_fused_dots_on_the_acoustic_operator():
    """The scalar acoustic operator's last pass forms the same inner products:
    BiCGStab and MixedBiCGStab on the 16^3 sphere scene follow the iterations
    of the separate alpha and omega kernels."""
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea
    from em3d_b200.solvers import BiCGStab, MixedBiCGStab, SolverConfig

    g = golden("ac_spheres16.npz")
    be = e.Backend.b200(e.Precision.DOUBLE)
    grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    prob = ea.make_acoustic_problem(grid, g["eta_double"], k0=20.0)
    op = ea.AcousticOperator(prob)
    lo = op.with_precision(e.Precision.SINGLE)
    assert op.dot_parts() > 0
    rhs = ea.plane_wave_scalar(grid, k=20.0, direction=(0.6, 0.8, 0.0))
    cfg = SolverConfig(max_iter=300, rtol=1e-8)
    runs = {}
    for fuse in (True, False):
        b = BiCGStab(cfg)
        b.fuse_dots = fuse
        m = MixedBiCGStab(cfg)
        m.fuse_dots = fuse
        runs[fuse] = (b.solve(op, rhs), m.solve(op, rhs, operator_low=lo))
    for k in range(2):
        a, c = runs[True][k], runs[False][k]
        assert a.status == c.status == "converged"
        assert a.iterations == c.iterations and a.matvec_count == c.matvec_count
        assert rel_err(be.to_host(a.u), be.to_host(c.u)) < 1e-7
