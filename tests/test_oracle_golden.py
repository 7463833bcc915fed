"""Pin the CPU oracle against golden vectors produced by the reference itself.

The fixtures come from ``tests/golden/make_golden.py``, which runs the
unmodified reference on the same seeded inputs.  These tests run on CPU.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_err
from oracle import acoustic as oac
from oracle import em as oem
from oracle import solvers as osol


@pytest.mark.parametrize("tag", ["4x3x3", "4x3x2", "5x6x7"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_em_kernel_hat_matches_reference(tag, prec):
    g = golden(f"em_kernel_hat_{tag}.npz")
    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    tol = 1e-13 if prec == "double" else 1e-6
    kh = oem.kernel_hat(N, L, k, prec)
    assert kh.dtype == g[f"kernel_hat_{prec}"].dtype
    assert rel_err(kh, g[f"kernel_hat_{prec}"]) < tol
    kha = oem.kernel_hat(N, L, k, prec, adjoint=True)
    assert rel_err(kha, g[f"kernel_hat_adjoint_{prec}"]) < tol


def test_em_self_term_is_minus_one_third():
    """Reference ``tests/test_operator_vs_dense.py:20-25``."""
    K = oem.kernel_blocks((4, 4, 4), (1.0, 1.0, 1.0), 1.0)
    np.testing.assert_allclose(K[:, :, 0, 0, 0], (-1.0 / 3.0) * np.eye(3), atol=1e-14)
    assert abs(K[0, 1, 1, 1, 0]) > 0.0


@pytest.mark.parametrize("case", ["sphere16", "cyl_lossy4", "aniso12", "odd567"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_em_matvec_rmatvec_match_reference(case, prec):
    g = golden(f"em_{case}.npz")
    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    tol = 1e-13 if prec == "double" else 2e-6
    chi, u = g[f"chi_{prec}"], g[f"u_{prec}"]
    kh = oem.kernel_hat(N, L, k, prec)
    kha = oem.kernel_hat(N, L, k, prec, adjoint=True)
    assert rel_err(oem.matvec(chi, u, kh, N), g[f"matvec_u_{prec}"]) < tol
    assert rel_err(oem.matvec(chi, g[f"wave_{prec}"], kh, N), g[f"matvec_wave_{prec}"]) < tol
    assert rel_err(oem.rmatvec(chi, u, N, khat_adjoint=kha), g[f"rmatvec_u_{prec}"]) < tol
    assert rel_err(oem.rmatvec(chi, u, N, khat=kh), g[f"rmatvec_u_derived_{prec}"]) < tol


def test_em_fft_matvec_matches_dense_known_answer():
    """Reference ``tests/test_operator_vs_dense.py:133-168`` (rel < 1e-10)."""
    g = golden("em_cyl_lossy4.npz")
    A = golden("em_dense_cyl_lossy4.npz")["A"]
    N, L, k = (4, 4, 4), (1.0, 1.0, 1.0), 1.0
    chi, u = g["chi_double"], g["u_double"]
    A_oracle = oem.dense_operator_matrix(chi, N, L, (0.0, 0.0, 0.0), k)
    assert rel_err(A_oracle, A) < 1e-13
    kh = oem.kernel_hat(N, L, k)
    y = oem.flatten_field(oem.matvec(chi, u, kh, N))
    assert rel_err(y, A @ oem.flatten_field(u)) < 1e-10
    ya = oem.flatten_field(oem.rmatvec(chi, u, N, khat=kh))
    assert rel_err(ya, A.conj().T @ oem.flatten_field(u)) < 1e-10


def test_crop_equivalent_kernel_gives_identical_matvec():
    """The symmetric spectrum the GPU path stores leaves the cropped operator unchanged."""
    g = golden("em_odd567.npz")
    N, L, k = (5, 6, 7), (1.0, 0.8, 1.3), 3.3
    chi, u = g["chi_double"], g["u_double"]
    Ksym = oem.kernel_blocks_crop_equivalent(N, L, k)
    kh_sym = np.fft.fftn(Ksym, axes=(-3, -2, -1))
    assert rel_err(oem.matvec(chi, u, kh_sym, N), g["matvec_u_double"]) < 1e-13
    assert rel_err(oem.rmatvec(chi, u, N, khat=kh_sym), g["rmatvec_u_double"]) < 1e-13
    # every block is now even (diagonal) or odd in its two axes: K_hat(-k) = K_hat(k)
    assert rel_err(oem.reverse_frequency_axes(kh_sym), kh_sym) < 1e-13


@pytest.mark.parametrize("case", ["sphere332", "spheres16", "odd765"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_acoustic_matvec_rmatvec_match_reference(case, prec):
    g = golden(f"ac_{case}.npz")
    N, L, k0 = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k0"])
    tol = 1e-13 if prec == "double" else 2e-6
    chi = (g[f"eta_{prec}"] - 1.0).astype(g[f"eta_{prec}"].dtype)
    u = g[f"u_{prec}"]
    kh = oac.kernel_hat(N, L, k0, prec)
    khc = oac.kernel_hat(N, L, k0, prec, adjoint=True)
    assert rel_err(oac.matvec(chi, u, kh, N), g[f"matvec_u_{prec}"]) < tol
    assert rel_err(oac.rmatvec(chi, u, khc, N), g[f"rmatvec_u_{prec}"]) < tol
    dv = oem.cell_volume(N, L)
    assert abs(oac.self_cell_coefficient(k0, dv) - complex(g[f"self_cell_{prec}"])) < 1e-15
    if g[f"kernel_{prec}"].size:
        assert rel_err(oac.kernel_on_doubled_grid(N, L, k0, prec), g[f"kernel_{prec}"]) < tol


def test_acoustic_dense_known_answer():
    """Reference ``tests/test_acoustics_operator.py:236-254`` (FFT == dense at 1e-12)."""
    g = golden("ac_sphere332.npz")
    N, L, k0 = (3, 3, 2), (1.0, 0.8, 0.6), 1.2
    chi = g["eta_double"] - 1.0
    H = oac.dense_operator_matrix(chi, N, L, (0.0, 0.0, 0.0), k0)
    u = g["u_double"]
    assert np.allclose(H @ u.reshape(-1), g["matvec_u_double"].reshape(-1), rtol=1e-12, atol=1e-12)


def _sphere16(prec):
    g = golden("em_sphere16.npz")
    N = (16, 16, 16)
    kh = oem.kernel_hat(N, (1.0, 1.0, 1.0), 4.0, prec)
    chi = g[f"chi_{prec}"]
    return g, N, kh, chi


@pytest.mark.parametrize("prec", ["double", "single"])
@pytest.mark.parametrize("solver", ["bicgstab", "twostep", "sim"])
def test_solvers_match_reference_histories(solver, prec):
    g, N, kh, chi = _sphere16(prec)
    sol = golden("solvers.json")
    ref = sol[f"sphere16_{solver}_{prec}"]
    rtol = 1e-8 if prec == "double" else 1e-5
    mv = lambda x: oem.matvec(chi, x, kh, N)  # noqa: E731
    khc = oem.kernel_hat(N, (1.0, 1.0, 1.0), 4.0, prec, adjoint=True)
    rmv = lambda x: oem.rmatvec(chi, x, N, khat_adjoint=khc)  # noqa: E731
    rhs = g[f"wave_{prec}"]
    if solver == "bicgstab":
        out = osol.bicgstab(mv, rhs, max_iter=200, rtol=rtol)
    elif solver == "twostep":
        out = osol.twostep(mv, rmv, rhs, max_iter=200, rtol=rtol)
    else:
        mu = complex(*sol[f"sphere16_gamma0_{prec}"]["mu"])
        out = osol.sim(mv, rhs, mu=mu, max_iter=200, rtol=rtol)
    assert out["status"] == ref["status"]
    assert out["iterations"] == ref["iterations"]
    assert out["matvec_count"] == ref["matvec_count"]
    assert out["rmatvec_count"] == ref["rmatvec_count"]
    assert out["residual_action_counts"] == ref["residual_action_counts"]
    htol = 1e-9 if prec == "double" else 1e-3
    np.testing.assert_allclose(out["residual_history"], ref["residual_history"], rtol=htol)
    u_ref = golden(f"sol_sphere16_{solver}_{prec}_u.npy")
    assert rel_err(out["u"], u_ref) < (1e-10 if prec == "double" else 1e-4)


@pytest.mark.parametrize("budget", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("solver", ["bicgstab", "twostep", "sim"])
def test_solver_action_budgets_match_reference(solver, budget):
    """Reference ``tests/test_solvers.py:154-176`` extended to budgets 1..5."""
    from em3d_b200.setup import cylinder_refraction, flat_wave_vec_host, grid_axes_host

    N, L, k = (4, 4, 4), (1.0, 1.0, 1.0), 0.5
    axes = grid_axes_host(N, L, (0.0, 0.0, 0.0), "double")
    chi = cylinder_refraction(axes, eps_real=1.1, eps_imag=0.0, radius=0.2, axis="z", dtype=np.complex128)
    wave = flat_wave_vec_host(axes, k=k, orient=(0, 0, 1), amplitude=(1, 0, 0), dtype=np.complex128)
    kh = oem.kernel_hat(N, L, k)
    khc = oem.kernel_hat(N, L, k, adjoint=True)
    mv = lambda x: oem.matvec(chi, x, kh, N)  # noqa: E731
    rmv = lambda x: oem.rmatvec(chi, x, N, khat_adjoint=khc)  # noqa: E731
    ref = golden("solvers.json")[f"budget{budget}_{solver}"]
    if solver == "bicgstab":
        out = osol.bicgstab(mv, wave, max_iter=100, max_operator_actions=budget)
    elif solver == "twostep":
        out = osol.twostep(mv, rmv, wave, max_iter=100, max_operator_actions=budget)
    else:
        out = osol.sim(mv, wave, mu=2.0 + 0j, max_iter=100, max_operator_actions=budget)
    for key in ("status", "iterations", "matvec_count", "rmatvec_count", "residual_action_counts"):
        assert out[key] == ref[key], key
    np.testing.assert_allclose(out["residual_history"], ref["residual_history"], rtol=1e-10)


def test_twostep_two_update_recurrence():
    """Reference ``tests/test_solvers.py:110-119`` (hand-written 2x2 recurrence, 1e-12)."""
    A = np.array([[2.0, 0.5], [1.0, 1.5]], dtype=np.complex128)
    rhs = np.array([1.0, -0.5], dtype=np.complex128)
    out = osol.twostep(lambda x: A @ x, lambda x: A.conj().T @ x, rhs, max_iter=2, rtol=1e-15)
    u0 = np.zeros(2, complex)
    r0 = A @ u0 - rhs
    g0 = A.conj().T @ r0
    Hg0 = A @ g0
    u1 = u0 - (np.vdot(g0, g0).real / np.vdot(Hg0, Hg0).real) * g0
    r1 = A @ u1 - rhs
    g1 = A.conj().T @ r1
    Hg1 = A @ g1
    dr = r1 - r0
    a00, a01, a11 = np.vdot(dr, dr).real, np.vdot(dr, Hg1).real, np.vdot(Hg1, Hg1).real
    b0, b1 = np.vdot(r1, dr).real, np.vdot(r1, Hg1).real
    det = a00 * a11 - a01 * a01
    t, h = (b0 * a11 - b1 * a01) / det, (a00 * b1 - a01 * b0) / det
    assert np.allclose(out["u"], u1 - t * (u1 - u0) - h * g1, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("case", ["aniso12", "odd567", "sphere16"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_streamed_em_oracle_matches_reference(case, prec):
    """The block-at-a-time oracle (used at 96^3 and 128^3 on the GPU box)
    against the reference's own matvec / explicit-adjoint rmatvec."""
    g = golden(f"em_{case}.npz")
    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    tol = 1e-13 if prec == "double" else 2e-6
    chi, u = g[f"chi_{prec}"], g[f"u_{prec}"]
    assert rel_err(oem.matvec_streamed(chi, u, N, L, k, precision=prec), g[f"matvec_u_{prec}"]) < tol
    assert rel_err(oem.matvec_streamed(chi, u, N, L, k, adjoint=True, precision=prec),
                   g[f"rmatvec_u_{prec}"]) < tol


@pytest.mark.parametrize("case", ["sphere332", "spheres16", "odd765"])
def test_streamed_acoustic_oracle_matches_reference(case):
    """The lean acoustic oracle (used at 256^3 on the GPU box) against the
    reference's own matvec and rmatvec."""
    g = golden(f"ac_{case}.npz")
    N, L, k0 = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k0"])
    chi = g["eta_double"] - 1.0
    u = g["u_double"]
    assert rel_err(oac.matvec_streamed(chi, u, N, L, k0), g["matvec_u_double"]) < 1e-13
    assert rel_err(oac.matvec_streamed(chi, u, N, L, k0, adjoint=True), g["rmatvec_u_double"]) < 1e-13
