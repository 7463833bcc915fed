"""Parity of the B200 operators with the reference (golden vectors) and the oracle.

Tolerances (relative 2-norm): FP64 path <= 1e-12, FP32 path <= 1e-5 against
the reference's own complex128 / complex64 results on the same inputs.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

TOL = {"double": 1e-12, "single": 1e-5}


def _be(prec):
    import em3d_b200 as e

    return e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)


def _em_problem(g, prec):
    import em3d_b200 as e

    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    be = _be(prec)
    grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
    prob = e.Problem(grid=grid, eps_tensor=g[f"chi_{prec}"], wave=g[f"wave_{prec}"], k0=k,
                     volume=grid.dv * int(np.prod(N)))
    return be, grid, prob


@pytest.mark.parametrize("case", ["sphere16", "cyl_lossy4", "aniso12", "odd567"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_em_matvec_rmatvec_match_reference(case, prec):
    import em3d_b200 as e

    g = golden(f"em_{case}.npz")
    be, grid, prob = _em_problem(g, prec)
    op = e.Operator(prob)
    u = g[f"u_{prec}"]
    y = be.to_host(op.matvec(u))
    assert y.dtype == g[f"matvec_u_{prec}"].dtype
    assert rel_err(y, g[f"matvec_u_{prec}"]) < TOL[prec]
    assert rel_err(be.to_host(op.matvec(g[f"wave_{prec}"])), g[f"matvec_wave_{prec}"]) < TOL[prec]
    assert rel_err(be.to_host(op.rmatvec(u)), g[f"rmatvec_u_{prec}"]) < TOL[prec]
    pk = e.PreparedEMKernel.build(grid, k=prob.k0, adjoint_storage="derived", build_strategy="streamed")
    op_d = e.Operator(prob, prepared_kernel=pk)
    assert rel_err(be.to_host(op_d.rmatvec(u)), g[f"rmatvec_u_derived_{prec}"]) < TOL[prec]


@pytest.mark.parametrize("case", ["sphere16", "aniso12"])
def test_fp32_path_against_reference_double(case):
    """The FP32 operator against the reference complex128 result (north-star bar 1e-5)."""
    import em3d_b200 as e

    g = golden(f"em_{case}.npz")
    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    be = _be("single")
    grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
    prob = e.Problem(grid=grid, eps_tensor=g["chi_double"].astype(np.complex64),
                     wave=g["wave_double"].astype(np.complex64), k0=k, volume=1.0)
    op = e.Operator(prob)
    y = be.to_host(op.matvec(g["u_double"].astype(np.complex64)))
    assert rel_err(y, g["matvec_u_double"]) < 1e-5


@pytest.mark.parametrize("tag", ["4x3x3", "4x3x2", "5x6x7"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_em_kernel_hat_full_matches_reference(tag, prec):
    import em3d_b200 as e

    g = golden(f"em_kernel_hat_{tag}.npz")
    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    be = _be(prec)
    grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
    pk = e.PreparedEMKernel.build(grid, k=k)
    tol = 1e-12 if prec == "double" else 1e-5
    assert rel_err(be.to_host(pk.kernel_hat), g[f"kernel_hat_{prec}"]) < tol
    assert rel_err(be.to_host(pk.kernel_hat_adjoint), g[f"kernel_hat_adjoint_{prec}"]) < tol
    pk.release_full_spectra()  # the octant alone is what the operator keeps
    assert pk.persistent_nbytes < g[f"kernel_hat_{prec}"].nbytes


def test_batched_matvec_equals_single():
    import torch
    import em3d_b200 as e

    g = golden("em_aniso12.npz")
    be, grid, prob = _em_problem(g, "double")
    op = e.Operator(prob)
    rng = np.random.default_rng(0)
    U = (rng.standard_normal((5, 3) + grid.N) + 1j * rng.standard_normal((5, 3) + grid.N)).astype(np.complex128)
    Y = be.to_host(op.matvec(U))
    for b in range(5):
        assert rel_err(Y[b], be.to_host(op.matvec(U[b]))) < 1e-14
    Ya = be.to_host(op.rmatvec(U))
    assert rel_err(Ya[2], be.to_host(op.rmatvec(U[2]))) < 1e-14
    del torch


def test_adjoint_identity_em():
    import em3d_b200 as e

    g = golden("em_odd567.npz")
    be, grid, prob = _em_problem(g, "double")
    op = e.Operator(prob)
    rng = np.random.default_rng(4)
    u = rng.standard_normal((3,) + grid.N) + 1j * rng.standard_normal((3,) + grid.N)
    v = rng.standard_normal((3,) + grid.N) + 1j * rng.standard_normal((3,) + grid.N)
    left = np.vdot(be.to_host(op.matvec(u)), v)
    right = np.vdot(u, be.to_host(op.rmatvec(v)))
    assert abs(left - right) < 1e-12 * abs(left)


def test_prepared_kernel_rejects_incompatible_wave_number():
    import em3d_b200 as e

    g = golden("em_cyl_lossy4.npz")
    be, grid, prob = _em_problem(g, "double")
    pk = e.PreparedEMKernel.build(grid, k=2.0)
    with pytest.raises(ValueError, match="wave number"):
        e.Operator(prob, prepared_kernel=pk)


def test_forward_only_kernel_rejects_adjoint_action():
    import em3d_b200 as e

    g = golden("em_cyl_lossy4.npz")
    be, grid, prob = _em_problem(g, "double")
    pk = e.PreparedEMKernel.build(grid, k=prob.k0, include_adjoint=False, build_strategy="streamed")
    op = e.Operator(prob, prepared_kernel=pk)
    with pytest.raises(RuntimeError, match="adjoint action is unavailable"):
        op.rmatvec(prob.wave)


def test_em_matvec_against_oracle_random_sizes():
    """Mixed-radix sizes the golden set does not cover, checked against the oracle live."""
    import em3d_b200 as e
    from oracle import em as oem

    rng = np.random.default_rng(12)
    for N, L, k in (((6, 10, 9), (1.1, 0.9, 1.0), 2.5), ((8, 12, 16), (1.0, 1.0, 1.0), 7.0),
                    ((24, 20, 15), (1.0, 1.2, 0.8), 5.0)):
        be = _be("double")
        grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
        chi = (rng.standard_normal((3, 3) + N) + 1j * rng.standard_normal((3, 3) + N)) * 0.3
        u = rng.standard_normal((3,) + N) + 1j * rng.standard_normal((3,) + N)
        prob = e.Problem(grid=grid, eps_tensor=chi, wave=u, k0=k, volume=1.0)
        op = e.Operator(prob)
        kh = oem.kernel_hat(N, L, k)
        assert rel_err(be.to_host(op.matvec(u)), oem.matvec(chi, u, kh, N)) < 1e-12
        assert rel_err(be.to_host(op.rmatvec(u)), oem.rmatvec(chi, u, N, khat=kh)) < 1e-12


@pytest.mark.parametrize("case", ["sphere332", "spheres16", "odd765"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_acoustic_matvec_rmatvec_match_reference(case, prec):
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea

    g = golden(f"ac_{case}.npz")
    N, L, k0 = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k0"])
    be = _be(prec)
    grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
    prob = ea.make_acoustic_problem(grid, g[f"eta_{prec}"], k0=k0)
    assert rel_err(be.to_host(prob.wave), g[f"wave_{prec}"]) < (1e-15 if prec == "double" else 1e-7)
    op = ea.AcousticOperator(prob)
    u = g[f"u_{prec}"]
    assert rel_err(be.to_host(op.matvec(u)), g[f"matvec_u_{prec}"]) < TOL[prec]
    assert rel_err(be.to_host(op.rmatvec(u)), g[f"rmatvec_u_{prec}"]) < TOL[prec]


def test_acoustic_identity_for_eta_one():
    """Reference ``tests/test_acoustics_operator.py:257-263``."""
    import torch
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea

    be = _be("double")
    grid = e.Grid(N=(3, 2, 2), L=(1.0, 0.8, 0.6), center=(0.0, 0.0, 0.0), backend=be)
    prob = ea.make_acoustic_problem(grid, ea.eta_homogeneous(grid, 1.0), k0=1.0)
    op = ea.AcousticOperator(prob)
    u = torch.ones(grid.N, dtype=torch.complex128, device="cuda") * (2.0 - 0.5j)
    assert torch.allclose(op.matvec(u), u)
    assert torch.allclose(op.rmatvec(u), u)


@pytest.mark.parametrize("prec", ["double", "single"])
@pytest.mark.parametrize("kind", ["em", "acoustic"])
def test_register_fft_path_matches_generic_path(prec, kind, monkeypatch):
    """The register-resident FFT passes (power-of-two doubled axes) against the
    generic shared-memory Stockham passes on the same inputs."""
    import torch
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea

    be = _be(prec)
    rng = np.random.default_rng(3)
    tol = 1e-13 if prec == "double" else 3e-6
    for N in ((32, 16, 64), (64, 64, 64), (128, 128, 128)) if kind == "em" else ((32, 64, 16), (128, 128, 128), (256, 128, 64)):
        grid = e.Grid(N=N, L=(1.0, 0.9, 1.1), center=(0.0, 0.0, 0.0), backend=be)
        tc = be.precision.torch_complex
        if kind == "em":
            chi = (torch.randn((3, 3) + N, dtype=tc, device="cuda") * 0.3).contiguous()
            u = torch.randn((3,) + N, dtype=tc, device="cuda")
            op = e.Operator(e.Problem(grid=grid, eps_tensor=chi, wave=u, k0=7.0, volume=1.0))
        else:
            eta = (1.0 + torch.rand(N, dtype=tc, device="cuda")).contiguous()
            op = ea.AcousticOperator(ea.make_acoustic_problem(grid, eta, k0=9.0))
            u = torch.randn(N, dtype=tc, device="cuda")
        from em3d_b200 import _lib
        from em3d_b200.tune import set_xpass_variant

        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FFT_GENERIC, 1)
        gen_mv, gen_rmv = op.matvec(u), op.rmatvec(u)
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FFT_GENERIC, 0)
        for v in (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10):
            set_xpass_variant(v)
            fast_mv, fast_rmv = op.matvec(u), op.rmatvec(u)
            assert rel_err(be.to_host(fast_mv), be.to_host(gen_mv)) < tol, (N, v)
            assert rel_err(be.to_host(fast_rmv), be.to_host(gen_rmv)) < tol, (N, v)
        set_xpass_variant(-1)
    del rng


@pytest.mark.parametrize("prec", ["double", "single"])
@pytest.mark.parametrize("kind", ["em", "acoustic"])
def test_mixed_radix_register_path_matches_generic_path(prec, kind):
    """Doubled axes 96 = 3 x 32, 160 = 5 x 32 and 192 = 3 x 64 on the register
    FFT (radix 4, 6 / 10 / 12, 4), every x-pass variant, against the generic
    passes (complex128 runs the x pass of 160 on the generic passes)."""
    import torch
    import em3d_b200 as e
    from em3d_b200 import _lib, acoustics as ea
    from em3d_b200.tune import set_xpass_variant

    be = _be(prec)
    tol = 1e-13 if prec == "double" else 3e-6
    for N in ((48, 80, 96), (96, 48, 16), (80, 96, 48)):
        grid = e.Grid(N=N, L=(1.0, 0.9, 1.1), center=(0.0, 0.0, 0.0), backend=be)
        tc = be.precision.torch_complex
        if kind == "em":
            chi = (torch.randn((3, 3) + N, dtype=tc, device="cuda") * 0.3).contiguous()
            u = torch.randn((3,) + N, dtype=tc, device="cuda")
            op = e.Operator(e.Problem(grid=grid, eps_tensor=chi, wave=u, k0=7.0, volume=1.0))
        else:
            eta = (1.0 + torch.rand(N, dtype=tc, device="cuda")).contiguous()
            op = ea.AcousticOperator(ea.make_acoustic_problem(grid, eta, k0=9.0))
            u = torch.randn(N, dtype=tc, device="cuda")
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FFT_GENERIC, 1)
        gen_mv, gen_rmv = op.matvec(u), op.rmatvec(u)
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FFT_GENERIC, 0)
        try:
            for v in (-1, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10):
                set_xpass_variant(v)
                fast_mv, fast_rmv = op.matvec(u), op.rmatvec(u)
                assert rel_err(be.to_host(fast_mv), be.to_host(gen_mv)) < tol, (N, v)
                assert rel_err(be.to_host(fast_rmv), be.to_host(gen_rmv)) < tol, (N, v)
        finally:
            set_xpass_variant(-1)


def test_em_matvec_oracle_on_mixed_radix_axes():
    """Doubled axes 96, 32 and 160 against the oracle: complex128 to 1e-12,
    complex64 to 1e-5."""
    import em3d_b200 as e
    from oracle import em as oem

    N, L, k = (48, 16, 80), (1.0, 0.5, 1.2), 9.0
    rng = np.random.default_rng(11)
    chi = (rng.standard_normal((3, 3) + N) + 1j * rng.standard_normal((3, 3) + N)) * 0.2
    u = rng.standard_normal((3,) + N) + 1j * rng.standard_normal((3,) + N)
    kh = oem.kernel_hat(N, L, k)
    ref, ref_a = oem.matvec(chi, u, kh, N), oem.rmatvec(chi, u, N, khat=kh)
    for prec, tol in (("double", 1e-12), ("single", 1e-5)):
        be = _be(prec)
        cdt = be.complex_dtype
        grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
        op = e.Operator(e.Problem(grid=grid, eps_tensor=chi.astype(cdt), wave=u.astype(cdt), k0=k, volume=1.0))
        assert rel_err(be.to_host(op.matvec(u.astype(cdt))), ref) < tol, prec
        assert rel_err(be.to_host(op.rmatvec(u.astype(cdt))), ref_a) < tol, prec


def test_em_matvec_oracle_at_32_cubed_both_paths(monkeypatch):
    """Register path and generic path both against the oracle (FP64, 1e-12)."""
    import em3d_b200 as e
    from oracle import em as oem

    g = golden("em_aniso12.npz")
    N, L, k = (32, 32, 32), (1.0, 1.0, 1.0), 12.0
    rng = np.random.default_rng(8)
    chi = (rng.standard_normal((3, 3) + N) + 1j * rng.standard_normal((3, 3) + N)) * 0.2
    u = rng.standard_normal((3,) + N) + 1j * rng.standard_normal((3,) + N)
    be = _be("double")
    grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
    op = e.Operator(e.Problem(grid=grid, eps_tensor=chi, wave=u, k0=k, volume=1.0))
    kh = oem.kernel_hat(N, L, k)
    ref, ref_a = oem.matvec(chi, u, kh, N), oem.rmatvec(chi, u, N, khat=kh)
    from em3d_b200 import _lib

    for generic in (0, 1):
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FFT_GENERIC, generic)
        assert rel_err(be.to_host(op.matvec(u)), ref) < 1e-12
        assert rel_err(be.to_host(op.rmatvec(u)), ref_a) < 1e-12
    _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FFT_GENERIC, 0)
    del g


@pytest.mark.parametrize("N", [(16, 16, 16), (32, 16, 64)])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_batched_matvec_equals_single_register_path(N, prec):
    """Batched application on the register-FFT path (power-of-two axes)."""
    import torch
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea

    be = _be(prec)
    tc = be.precision.torch_complex
    grid = e.Grid(N=N, L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    gen = torch.Generator(device="cuda").manual_seed(1)
    chi = (torch.randn((3, 3) + N, dtype=tc, device="cuda", generator=gen) * 0.3).contiguous()
    U = torch.randn((7, 3) + N, dtype=tc, device="cuda", generator=gen)
    op = e.Operator(e.Problem(grid=grid, eps_tensor=chi, wave=U[0], k0=5.0, volume=1.0))
    tol = 1e-14 if prec == "double" else 1e-6
    from em3d_b200.tune import set_xpass_variant

    for v in (0, 3, 4, 7, 8):
        set_xpass_variant(v)
        Y, Ya = op.matvec(U), op.rmatvec(U)
        for b in range(7):
            assert rel_err(be.to_host(Y[b]), be.to_host(op.matvec(U[b]))) < tol, (v, b)
            assert rel_err(be.to_host(Ya[b]), be.to_host(op.rmatvec(U[b]))) < tol, (v, b)
    set_xpass_variant(-1)
    eta = (1.0 + torch.rand(N, dtype=tc, device="cuda", generator=gen)).contiguous()
    aop = ea.AcousticOperator(ea.make_acoustic_problem(grid, eta, k0=6.0))
    V = torch.randn((5,) + N, dtype=tc, device="cuda", generator=gen)
    Z = aop.matvec(V)
    for b in range(5):
        assert rel_err(be.to_host(Z[b]), be.to_host(aop.matvec(V[b]))) < tol, b


@pytest.mark.parametrize("prec", ["double", "single"])
def test_tma_field_slab_completes(prec):
    """The TMA-fed x-pass variants (5, 6) give the cp.async variants' result
    and no bounded wait gives up (the status word at the end of the apply
    workspace stays zero)."""
    import torch
    import em3d_b200 as e
    from em3d_b200.tune import set_xpass_variant

    be = _be(prec)
    tol = 1e-13 if prec == "double" else 3e-6
    for N in ((32, 16, 64), (64, 64, 64), (48, 96, 32)):
        grid = e.Grid(N=N, L=(1.0, 0.9, 1.1), center=(0.0, 0.0, 0.0), backend=be)
        tc = be.precision.torch_complex
        chi = (torch.randn((3, 3) + N, dtype=tc, device="cuda") * 0.3).contiguous()
        u = torch.randn((2, 3) + N, dtype=tc, device="cuda")
        op = e.Operator(e.Problem(grid=grid, eps_tensor=chi, wave=u[0], k0=7.0, volume=1.0))
        try:
            set_xpass_variant(3)
            ref, ref_a = op.matvec(u), op.rmatvec(u)
            for v in (5, 6, 7, 8, 9, 10):
                set_xpass_variant(v)
                assert rel_err(be.to_host(op.matvec(u)), be.to_host(ref)) < tol, (N, v)
                assert rel_err(be.to_host(op.rmatvec(u)), be.to_host(ref_a)) < tol, (N, v)
        finally:
            set_xpass_variant(-1)
        torch.cuda.synchronize()
        assert int(op.workspace(2)[-256:].view(torch.int32)[0]) == 0


def test_lost_transfer_count_raises_and_resets():
    """The give-up count at the end of the apply workspace (bounded waits on
    TMA transfers that never completed) turns into ``NativeError`` in the
    public matvec / rmatvec and in a solve.  The count is planted from the
    host; nothing is made to fail on the device."""
    import torch
    import em3d_b200 as e
    from em3d_b200 import _lib
    from em3d_b200.solvers import BiCGStab, MixedBiCGStab, SolverConfig

    g = golden("em_aniso12.npz")
    be, grid, prob = _em_problem(g, "double")
    op = e.Operator(prob)
    ref = op.matvec(prob.wave)
    for adjoint in (False, True):
        op.status_word(1).fill_(3)
        with pytest.raises(_lib.NativeError, match="3 bounded wait"):
            op.rmatvec(prob.wave) if adjoint else op.matvec(prob.wave)
        assert int(op.status_word(1).item()) == 0  # reset: the operator stays usable
    assert rel_err(be.to_host(op.matvec(prob.wave)), be.to_host(ref)) == 0.0
    # a solve reads the count together with its done flag
    op.status_word(1).fill_(1)
    with pytest.raises(_lib.NativeError, match="bounded wait"):
        BiCGStab(SolverConfig(max_iter=50, rtol=1e-8)).solve(op, prob.wave)
    op32 = op.with_precision(e.Precision.SINGLE)
    op32.status_word(1).fill_(2)
    with pytest.raises(_lib.NativeError, match="bounded wait"):
        MixedBiCGStab(SolverConfig(max_iter=50, rtol=1e-8)).solve(op, prob.wave, operator_low=op32)
    res = MixedBiCGStab(SolverConfig(max_iter=50, rtol=1e-8)).solve(op, prob.wave, operator_low=op32)
    assert res.converged
    torch.cuda.synchronize()


@pytest.mark.parametrize("kind", ["em", "acoustic"])
def test_fp32_twin_spectrum_is_the_complex64_build(kind):
    """``with_precision`` rounds the FP64 spectrum instead of rebuilding it;
    the bytes equal those of a complex64 build."""
    import torch
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea

    N = (12, 10, 16)
    be64, be32 = _be("double"), _be("single")
    g64 = e.Grid(N=N, L=(1.0, 0.9, 1.1), center=(0.0, 0.0, 0.0), backend=be64)
    g32 = e.Grid(N=N, L=(1.0, 0.9, 1.1), center=(0.0, 0.0, 0.0), backend=be32)
    if kind == "em":
        chi = torch.randn((3, 3) + N, dtype=torch.complex128, device="cuda") * 0.3
        u = torch.randn((3,) + N, dtype=torch.complex128, device="cuda")
        op64 = e.Operator(e.Problem(grid=g64, eps_tensor=chi, wave=u, k0=7.0, volume=1.0))
        twin = op64.with_precision(e.Precision.SINGLE)
        built = e.PreparedEMKernel.build(g32, k=7.0)
        assert torch.equal(twin.prepared_kernel.spectrum, built.spectrum)
        assert twin.prepared_kernel.precision == "single"
    else:
        eta = (1.0 + torch.rand(N, dtype=torch.complex128, device="cuda")).contiguous()
        op64 = ea.AcousticOperator(ea.make_acoustic_problem(g64, eta, k0=9.0))
        twin = op64.with_precision(e.Precision.SINGLE)
        built = ea.AcousticOperator(ea.make_acoustic_problem(g32, eta.to(torch.complex64), k0=9.0))
        assert torch.equal(twin._spectrum, built._spectrum)
        u = torch.randn(N, dtype=torch.complex128, device="cuda")
    y64 = op64.matvec(u)
    y32 = twin.matvec(u.to(be32.precision.torch_complex))
    assert rel_err(be32.to_host(y32), be64.to_host(y64)) < 1e-5


def test_persistent_nbytes_counts_materialised_full_spectra():
    import em3d_b200 as e

    g = golden("em_kernel_hat_4x3x3.npz")
    N, L, k = tuple(int(v) for v in g["N"]), tuple(float(v) for v in g["L"]), float(g["k"])
    grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=_be("double"))
    pk = e.PreparedEMKernel.build(grid, k=k)
    octant = pk.persistent_nbytes
    full = pk.kernel_hat
    assert pk.persistent_nbytes == octant + full.numel() * full.element_size()
    pk.kernel_hat_adjoint
    assert pk.persistent_nbytes == octant + 2 * full.numel() * full.element_size()
    pk.release_full_spectra()
    assert pk.persistent_nbytes == octant


@pytest.mark.parametrize("N", [(32, 16, 32), (12, 10, 9)])
@pytest.mark.parametrize("kind", ["isotropic", "symmetric", "full"])
def test_compact_contrast_storage_against_oracle(kind, N):
    """The operator stores an isotropic contrast as one value per cell and a
    symmetric one as six; matvec and rmatvec still equal the oracle's on the
    full tensor (register passes at (32,16,32), generic at (12,10,9))."""
    import em3d_b200 as e
    from oracle import em as oem

    rng = np.random.default_rng(21)
    L, k = (1.0, 0.8, 1.2), 5.5
    s = (rng.standard_normal(N) + 1j * rng.standard_normal(N)) * 0.4
    if kind == "isotropic":
        chi = np.einsum("ab,...->ab...", np.eye(3), s)
    else:
        chi = (rng.standard_normal((3, 3) + N) + 1j * rng.standard_normal((3, 3) + N)) * 0.3
        if kind == "symmetric":
            chi = 0.5 * (chi + chi.swapaxes(0, 1))
    u = rng.standard_normal((3,) + N) + 1j * rng.standard_normal((3,) + N)
    kh = oem.kernel_hat(N, L, k)
    ref, ref_a = oem.matvec(chi, u, kh, N), oem.rmatvec(chi, u, N, khat=kh)
    for prec, tol in (("double", 1e-12), ("single", 1e-5)):
        be = _be(prec)
        cdt = be.complex_dtype
        grid = e.Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
        op = e.Operator(e.Problem(grid=grid, eps_tensor=chi.astype(cdt), wave=u.astype(cdt), k0=k, volume=1.0))
        assert op.chi_layout == kind
        assert rel_err(be.to_host(op.matvec(u.astype(cdt))), ref) < tol, prec
        assert rel_err(be.to_host(op.rmatvec(u.astype(cdt))), ref_a) < tol, prec
