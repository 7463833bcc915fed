"""The host input builders reproduce the reference's inputs bit for bit (CPU)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from em3d_b200 import setup as S
from em3d_b200 import workloads as W


@pytest.mark.parametrize("prec", ["double", "single"])
def test_sphere_and_wave_match_reference(prec):
    g = golden("em_sphere16.npz")
    case = W.sphere_em(16, prec)
    np.testing.assert_array_equal(case.chi, g[f"chi_{prec}"])
    np.testing.assert_array_equal(case.wave, g[f"wave_{prec}"])


@pytest.mark.parametrize("prec", ["double", "single"])
def test_rotated_anisotropic_ellipsoid_matches_reference(prec):
    g = golden("em_aniso12.npz")
    rot = golden("em_rotation_seed0.npz")
    np.testing.assert_allclose(W.aniso_permittivity(0), rot["eps_aniso"], rtol=0, atol=0)
    case = W.aniso_ellipsoid_em(12, prec)
    np.testing.assert_array_equal(case.chi, g[f"chi_{prec}"])
    np.testing.assert_array_equal(case.wave, g[f"wave_{prec}"])


def test_odd_grid_inputs_match_reference():
    g = golden("em_odd567.npz")
    N, L = (5, 6, 7), (1.0, 0.8, 1.3)
    for prec in ("double", "single"):
        axes = S.grid_axes_host(N, L, (0.0, 0.0, 0.0), prec)
        cdt = S.complex_dtype_of(prec)
        chi = S.sample_contrast_tensor(axes, L, background_eps_r=1.0, feature_eps_r=W.aniso_permittivity(0),
                                       geometry=S.Ellipsoid((0.05, 0.0, -0.1), (0.45, 0.3, 0.5)), dtype=cdt)
        np.testing.assert_array_equal(chi, g[f"chi_{prec}"])
        wave = S.flat_wave_vec_host(axes, k=3.3, orient=(0.6, 0.0, 0.8), amplitude=(0, 1, 0), dtype=cdt)
        np.testing.assert_array_equal(wave, g[f"wave_{prec}"])


def test_cylinder_refraction_matches_reference():
    g = golden("em_cyl_lossy4.npz")
    for prec in ("double", "single"):
        axes = S.grid_axes_host((4, 4, 4), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), prec)
        chi = S.cylinder_refraction(axes, eps_real=2.0, eps_imag=0.5, radius=0.3, axis="z",
                                    dtype=S.complex_dtype_of(prec))
        np.testing.assert_array_equal(chi, g[f"chi_{prec}"])


def test_acoustic_inputs_match_reference():
    g = golden("ac_sphere332.npz")
    for prec in ("double", "single"):
        cdt = S.complex_dtype_of(prec)
        axes = S.grid_axes_host((3, 3, 2), (1.0, 0.8, 0.6), (0.0, 0.0, 0.0), prec)
        eta = S.eta_sphere(axes, center=(0.0, 0.0, 0.0), radius=0.45, eta_inside=2.0 + 0.2j, eta_outside=1.0,
                           dtype=cdt)
        np.testing.assert_array_equal(eta, g[f"eta_{prec}"])
        wave = S.plane_wave_scalar_host(axes, k=1.2, dtype=cdt)
        np.testing.assert_array_equal(wave, g[f"wave_{prec}"])


def test_input_validation_errors():
    axes = S.grid_axes_host((4, 4, 4), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    with pytest.raises(ValueError, match="unit vector"):
        S.flat_wave_vec_host(axes, k=1.0, orient=(1.0, 1.0, 0.0), amplitude=(1, 0, 0))
    with pytest.raises(ValueError, match="sign"):
        S.flat_wave_vec_host(axes, k=1.0, orient=(0, 0, 1), amplitude=(1, 0, 0), sign=2)
    with pytest.raises(ValueError, match="radii"):
        S.Ellipsoid((0, 0, 0), (0.1, -1.0, 0.1))
    with pytest.raises(ValueError, match="direction"):
        S.plane_wave_scalar_host(axes, k=1.0, direction=(0.0, 0.0, 0.0))


def test_multi_rhs_directions_and_polarisations():
    d = W.fibonacci_directions(64)
    assert d.shape == (64, 3)
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-12)
    assert abs(d[:, 2].mean()) < 1e-12  # symmetric spiral
    for v in d:
        p1, p2 = W.orthogonal_polarisations(v)
        assert abs(p1 @ v) < 1e-12 and abs(p2 @ v) < 1e-12 and abs(p1 @ p2) < 1e-12
    axes = S.grid_axes_host((6, 6, 6), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    waves = W.plane_wave_batch(axes, 10.0, 3)
    assert waves.shape == (6, 3, 6, 6, 6)


def test_acoustic_spheres_are_disjoint_and_seeded():
    a = W.acoustic_spheres(32, count=20, seed=0)
    b = W.acoustic_spheres(32, count=20, seed=0)
    np.testing.assert_array_equal(a.eta, b.eta)
    inside = a.eta != 1
    assert 0 < inside.mean() < 0.5
    vals = a.eta[inside]
    assert np.all((vals.real >= 1.2) & (vals.real <= 2.5) & (vals.imag >= 0) & (vals.imag <= 0.1))


def test_uneven_sphere_params():
    """The uneven-size set: seeded, every size present, parameters inside
    their ranges."""
    a = W.uneven_sphere_params(48, seed=0)
    assert a == W.uneven_sphere_params(48, seed=0)
    assert a != W.uneven_sphere_params(48, seed=1)
    assert sorted({p["N"] for p in a}) == [32, 48, 64, 80]
    for p in a:
        assert 0.15 <= p["radius"] <= 0.35 and 2.0 <= p["k0"] <= 8.0
        assert 1.5 <= p["eps"].real <= 4.0 and 0.0 <= p["eps"].imag <= 0.2
        assert p["orient"] == (0.0, 0.0, 1.0) and p["amplitude"] == (1.0, 0.0, 0.0)
