"""Parity at the benchmark's own sizes, against the oracle run live on the host.

The benchmark's numbers are measured on these configurations, so each is
checked directly against the CPU restatement of the reference (not against
another path of this library):

* the absorbing anisotropic ellipsoid at 128^3 (doubled axes 256, k0 = 12):
  EM matvec and rmatvec, complex128 (<= 1e-12) and complex64 (<= 1e-5 against
  the complex128 oracle), reference ``src/em3d/operator.py:353-398``;
* the same ellipsoid at 96^3 (doubled axes 192 = 3 x 64, k0 = 10);
* the 200-sphere acoustic scene at 256^3 (doubled axes 512, k0 = 20):
  matvec and rmatvec, reference ``src/em3d/acoustics/operator.py:40-67``;
* one full 128^3 mixed-precision solve to a true residual of 1e-6, whose
  residual is recomputed with the oracle's matvec on the host.

The oracle builds the kernel spectra one block at a time
(``oracle.em.matvec_streamed``); each 128^3 application takes a few seconds
on the host.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _em_operator(case, prec):
    import em3d_b200 as e

    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    cdt = be.complex_dtype
    grid = e.Grid(N=case.N, L=case.L, center=case.center, backend=be)
    prob = e.Problem(grid=grid, eps_tensor=case.chi.astype(cdt), wave=case.wave.astype(cdt), k0=case.k0,
                     volume=1.0)
    return be, e.Operator(prob)


def _random_field(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.fixture(scope="module")
def ellipsoid128():
    from em3d_b200 import workloads
    from oracle import em as oem

    case = workloads.aniso_ellipsoid_em(128, "double")
    u = _random_field((3,) + case.N, 128)
    ref = {
        "mv_u": oem.matvec_streamed(case.chi, u, case.N, case.L, case.k0),
        "rmv_u": oem.matvec_streamed(case.chi, u, case.N, case.L, case.k0, adjoint=True),
        "mv_wave": oem.matvec_streamed(case.chi, case.wave, case.N, case.L, case.k0),
    }
    return case, u, ref


@pytest.mark.parametrize("prec,tol", [("double", 1e-12), ("single", 1e-5)])
def test_em_128_matvec_rmatvec_against_oracle(ellipsoid128, prec, tol):
    case, u, ref = ellipsoid128
    be, op = _em_operator(case, prec)
    cdt = be.complex_dtype
    assert rel_err(be.to_host(op.matvec(u.astype(cdt))), ref["mv_u"]) < tol
    assert rel_err(be.to_host(op.rmatvec(u.astype(cdt))), ref["rmv_u"]) < tol
    assert rel_err(be.to_host(op.matvec(case.wave.astype(cdt))), ref["mv_wave"]) < tol


@pytest.mark.parametrize("prec,tol", [("double", 1e-12), ("single", 1e-5)])
def test_em_96_matvec_rmatvec_against_oracle(prec, tol):
    from em3d_b200 import workloads
    from oracle import em as oem

    case = workloads.aniso_ellipsoid_em(96, "double", k0=10.0)
    u = _random_field((3,) + case.N, 96)
    be, op = _em_operator(case, prec)
    cdt = be.complex_dtype
    ref = oem.matvec_streamed(case.chi, u, case.N, case.L, case.k0)
    ref_a = oem.matvec_streamed(case.chi, u, case.N, case.L, case.k0, adjoint=True)
    assert rel_err(be.to_host(op.matvec(u.astype(cdt))), ref) < tol
    assert rel_err(be.to_host(op.rmatvec(u.astype(cdt))), ref_a) < tol


@pytest.fixture(scope="module")
def acoustic256():
    from em3d_b200 import workloads
    from oracle import acoustic as oac

    case = workloads.acoustic_spheres(256, "double")
    chi = case.eta - 1.0
    u = _random_field(case.N, 256)
    ref = oac.matvec_streamed(chi, u, case.N, case.L, case.k0)
    ref_a = oac.matvec_streamed(chi, u, case.N, case.L, case.k0, adjoint=True)
    return case, u, ref, ref_a


@pytest.mark.parametrize("prec,tol", [("double", 1e-12), ("single", 1e-5)])
def test_acoustic_256_matvec_rmatvec_against_oracle(acoustic256, prec, tol):
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea

    case, u, ref, ref_a = acoustic256
    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    cdt = be.complex_dtype
    grid = e.Grid(N=case.N, L=case.L, center=case.center, backend=be)
    op = ea.AcousticOperator(ea.make_acoustic_problem(grid, case.eta.astype(cdt), k0=case.k0))
    assert rel_err(be.to_host(op.matvec(u.astype(cdt))), ref) < tol
    assert rel_err(be.to_host(op.rmatvec(u.astype(cdt))), ref_a) < tol


def test_device_sampled_acoustic_scene_matches_host_scene():
    """The benchmark samples the 200 spheres on the device; the parity test
    above uses the host builder.  Both give the same eta bit for bit."""
    import em3d_b200 as e
    from em3d_b200 import workloads

    be = e.Backend.b200(e.Precision.DOUBLE)
    grid = e.Grid(N=(256,) * 3, L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    dev = be.to_host(workloads.acoustic_spheres_device(grid, count=200, seed=0))
    host = workloads.acoustic_spheres(256, "double").eta
    assert np.array_equal(dev, host)


def test_mixed_solve_128_true_residual_by_oracle(ellipsoid128):
    """A full 128^3 mixed-precision solve (FP32 BiCGStab, FP64 reliable
    updates) to a true residual of 1e-6; the residual ||f - A u|| / ||f|| of
    its solution is recomputed on the host with the oracle's matvec."""
    import em3d_b200 as e
    from em3d_b200.solvers import MixedBiCGStab, SolverConfig
    from oracle import em as oem

    case, _, _ = ellipsoid128
    be, op64 = _em_operator(case, "double")
    op32 = op64.with_precision(e.Precision.SINGLE)
    res = MixedBiCGStab(SolverConfig(max_iter=500, rtol=1e-6)).solve(op64, op64.problem.wave, operator_low=op32)
    assert res.converged, res.status
    u = be.to_host(res.u)
    Au = oem.matvec_streamed(case.chi, u, case.N, case.L, case.k0)
    true_rel = np.linalg.norm((Au - case.wave).ravel()) / np.linalg.norm(case.wave.ravel())
    assert true_rel < 1e-6
    assert abs(true_rel - res.true_final_residual) < 1e-9
