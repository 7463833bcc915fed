"""Generate ``gamma0.json``: the reference's spectrum localisation and its
coarse-operator gamma0 estimates, by running the unmodified reference em3d.

    python tests/golden/make_gamma0_golden.py <reference checkout>/src

Spectrum cases are seeded point sets (clusters, a ring around the origin, two
points, a single repeated point); problem cases reuse the committed input
fixtures (``em_sphere16.npz``, ``em_aniso12.npz``, ``ac_spheres16.npz``).
Nothing at test time reads the reference; the tests read the JSON file.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def spectra():
    rng = np.random.default_rng(5)
    out = {
        "cluster": 1.5 + 0.3j + 0.4 * (rng.standard_normal(60) + 1j * rng.standard_normal(60)),
        "half_disc": 1.0 + 0.8 * np.exp(1j * rng.uniform(-1.2, 1.2, 40)) * rng.uniform(0, 1, 40),
        "ring_around_origin": np.exp(1j * np.linspace(0, 2 * np.pi, 12, endpoint=False)),
        "two_points": np.array([1.0 + 0.5j, 2.0 - 0.25j]),
        "repeated": np.array([1.0 + 1.0j] * 5),
        "far_left": -3.0 + 0.2j + 0.5 * (rng.standard_normal(30) + 1j * rng.standard_normal(30)),
    }
    return {k: np.asarray(v, dtype=np.complex128) for k, v in out.items()}


def main(ref_src: str) -> None:
    sys.path.insert(0, ref_src)
    import em3d
    from em3d import Backend, Grid, Precision, Problem, gamma0
    from em3d.acoustics import make_acoustic_problem
    from em3d.acoustics import gamma0 as ac_gamma0

    assert em3d.__version__ == "0.8.0", em3d.__version__
    res = {"spectra": {}, "problems": {}}
    for name, z in spectra().items():
        entry = {"points": [[v.real, v.imag] for v in z]}
        try:
            g = gamma0.analyze_spectrum(z)
            entry.update(mu=[g.mu.real, g.mu.imag], radius=g.radius, rho=g.rho,
                         hull=[[v.real, v.imag] for v in g.hull])
        except ValueError as exc:
            entry["error"] = str(exc)
        res["spectra"][name] = entry
    be = Backend.numpy(Precision.DOUBLE)
    for name, fixture, k_key in (("em_sphere16", "em_sphere16.npz", None), ("em_aniso12", "em_aniso12.npz", "k")):
        d = np.load(os.path.join(HERE, fixture))
        N = tuple(int(n) for n in d["N"])
        L = tuple(float(v) for v in d["L"])
        k0 = 4.0 if k_key is None else float(d[k_key])
        grid = Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be)
        prob = Problem(grid=grid, eps_tensor=d["chi_double"], wave=d["wave_double"], k0=k0, volume=1.0)
        for cn in ((4, 4, 4), (3, 4, 2)):
            key = f"{name}_coarse{''.join(map(str, cn))}"
            try:
                g = gamma0.estimate_from_problem(prob, coarse_N=cn)
                res["problems"][key] = {"mu": [g.mu.real, g.mu.imag], "radius": g.radius, "rho": g.rho}
            except ValueError as exc:
                res["problems"][key] = {"error": str(exc)}
    d = np.load(os.path.join(HERE, "ac_spheres16.npz"))
    grid = Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    for k0 in (20.0, 6.0):
        prob = make_acoustic_problem(grid, d["eta_double"], k0=k0)
        key = f"ac_spheres16_k{int(k0)}_coarse444"
        try:
            g = ac_gamma0.estimate_from_problem(prob, coarse_N=(4, 4, 4))
            res["problems"][key] = {"mu": [g.mu.real, g.mu.imag], "radius": g.radius, "rho": g.rho}
        except ValueError as exc:
            res["problems"][key] = {"error": str(exc)}
    with open(os.path.join(HERE, "gamma0.json"), "w") as fh:
        json.dump(res, fh, indent=1)
    for k, v in res["problems"].items():
        print(k, v)
    for k, v in res["spectra"].items():
        print(k, {kk: vv for kk, vv in v.items() if kk not in ("points", "hull")})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")
