"""SIM step size from the coarse operator's spectrum (``em3d_b200.gamma0``),
pinned to the reference's own localisation and estimates (``gamma0.json``,
generated by ``tests/golden/make_gamma0_golden.py``)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

G = golden("gamma0.json")


@pytest.mark.parametrize("name", sorted(G["spectra"]))
def test_spectrum_localisation_equals_reference(name):
    from em3d_b200 import gamma0

    case = G["spectra"][name]
    z = np.array([complex(a, b) for a, b in case["points"]])
    if "error" in case:
        with pytest.raises(ValueError, match=case["error"].split(":")[0]):
            gamma0.analyze_spectrum(z)
        return
    g = gamma0.analyze_spectrum(z)
    assert abs(g.mu - complex(*case["mu"])) < 1e-12 * max(1.0, abs(g.mu))
    assert abs(g.radius - case["radius"]) < 1e-12 * max(1.0, g.radius)
    assert abs(g.rho - case["rho"]) < 1e-12
    np.testing.assert_allclose(g.hull, [complex(a, b) for a, b in case["hull"]], rtol=0, atol=0)
    assert g.as_solver_config_kwargs() == {"mu": g.mu, "radius": g.radius}


def test_localisation_helpers():
    from em3d_b200 import gamma0

    mu, r = gamma0.circle_three_points(1 + 0j, 1j, -1 + 0j)
    assert abs(mu) < 1e-15 and abs(r - 1.0) < 1e-15
    with pytest.raises(ValueError):
        gamma0.circle_three_points(0j, 1 + 1j, 2 + 2j)
    # the two-point circle passes through both points
    mu, r = gamma0.circle_two_points(1 + 0.5j, 2 - 0.25j)
    assert abs(abs(1 + 0.5j - mu) - r) < 1e-12 and abs(abs(2 - 0.25j - mu) - r) < 1e-12
    assert gamma0.origin_in_hull(gamma0.convex_hull([1 + 1j, -1 + 1j, -1 - 1j, 1 - 1j]))
    assert not gamma0.origin_in_hull(gamma0.convex_hull([1 + 1j, 2 + 1j, 2 - 1j, 1 - 1j]))
    with pytest.raises(ValueError, match="coarse_N"):
        gamma0._shape((4, 4))


def _problem(name):
    import em3d_b200 as e
    from em3d_b200 import acoustics as ea

    be = e.Backend.b200(e.Precision.DOUBLE)
    if name.startswith("ac_"):
        d = golden("ac_spheres16.npz")
        grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
        k0 = float(name.split("_k")[1].split("_")[0])
        return ea.make_acoustic_problem(grid, d["eta_double"], k0=k0)
    fixture, k0 = ("em_sphere16.npz", 4.0) if name.startswith("em_sphere16") else ("em_aniso12.npz", None)
    d = golden(fixture)
    grid = e.Grid(N=tuple(int(n) for n in d["N"]), L=tuple(float(v) for v in d["L"]), center=(0.0, 0.0, 0.0),
                  backend=be)
    return e.Problem(grid=grid, eps_tensor=d["chi_double"], wave=d["wave_double"],
                     k0=k0 if k0 is not None else float(d["k"]), volume=1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(G["problems"]))
def test_estimate_from_problem_equals_reference(name):
    from em3d_b200 import gamma0

    case = G["problems"][name]
    cn = tuple(int(c) for c in name.split("coarse")[1])
    prob = _problem(name)
    if "error" in case:
        with pytest.raises(ValueError, match=case["error"].split(":")[0]):
            gamma0.estimate_from_problem(prob, coarse_N=cn)
        return
    g = gamma0.estimate_from_problem(prob, coarse_N=cn)
    assert abs(g.mu - complex(*case["mu"])) < 1e-9 * abs(g.mu)
    assert abs(g.radius - case["radius"]) < 1e-9 * max(g.radius, 1e-3)
    assert g.coarse_N == cn and g.matrix_shape[0] == g.matrix_shape[1]


@pytest.mark.gpu
def test_sim_runs_with_estimated_step():
    """SIM on the 16^3 sphere with mu and radius from the estimate converges
    like the reference's SIM with the reference's estimate."""
    import em3d_b200 as e
    from em3d_b200 import gamma0
    from em3d_b200.solvers import SIM, SolverConfig

    prob = _problem("em_sphere16_coarse444")
    g = gamma0.estimate_from_problem(prob)
    ref = golden("solvers.json")["sphere16_sim_double"]
    res = SIM(SolverConfig(max_iter=200, rtol=1e-8, **g.as_solver_config_kwargs())).solve(e.Operator(prob), prob.wave)
    assert res.status == ref["status"] and res.iterations == ref["iterations"]
